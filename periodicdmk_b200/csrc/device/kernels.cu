// CUDA kernels of the periodic DMK evaluate path, FP64 (plain) variant.
//
// Stage -> reference function it computes:
//   k_gather      charge gather into tree order (periodic_dmk.cpp:165-169, pbc_tree.cpp:1807-1821)
//   k_c2proxy     charge -> Chebyshev proxy moments (proxy.cpp:153-212)
//   k_contract    separable tensor transforms: c2p/p2c (tensorprod.cpp:39-75),
//                 proxy -> plane waves (proxy.cpp:42-90), plane waves -> proxy (planewave.cpp:49-105)
//   k_shift       plane-wave translation with the kernel FT fused (pbc_tree.cpp:1294-1348, tree.hpp:287-316)
//   k_eval        proxy -> potential at leaf targets (proxy.cpp:307-448)
//   k_near        PSWF residual pair sum (pbc_tree.cpp:1442-1681, vector_kernels.hpp:354-421)
//   k_spread / k_interp / k_multiply   periodic far field (pbc.cpp:359-541)
//   k_finalize    self correction + desort + far field add (pbc_tree.cpp:1759-1805, periodic_dmk.cpp:177-183)
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "kernels.cuh"

namespace pdmkb {
namespace dev {

// ============================================================================
// gather
// ============================================================================
__global__ void k_gather(double4* __restrict__ src, const int* __restrict__ idx, const double* __restrict__ q, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) src[i].w = q[idx[i]];
}

void launch_gather(double4* src, const int* src_charge_idx, const double* q_user, int n_all, cudaStream_t s) {
    if (n_all <= 0) return;
    k_gather<<<(n_all + 255) / 256, 256, 0, s>>>(src, src_charge_idx, q_user, n_all);
}

__global__ void k_gather_q(const int* __restrict__ perm, const double* __restrict__ q, double* __restrict__ out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = q[perm[i]];
}

void launch_nufft_gather_q(const int* trg_perm, const double* q_user, double* q_sorted, int n, cudaStream_t s) {
    if (n <= 0) return;
    k_gather_q<<<(n + 255) / 256, 256, 0, s>>>(trg_perm, q_user, q_sorted, n);
}

// ============================================================================
// charge -> proxy moments.  One CTA = one centre box x 128 (j,k) columns; each
// thread accumulates the P coefficients along x of its column over all sources.
// ============================================================================
template <int P>
__global__ void __launch_bounds__(128) k_c2proxy(C2ProxyArgs a) {
    constexpr int TS = 32;
    __shared__ double sx[TS][P], sy[TS][P], sz[TS][P];
    const int e = blockIdx.x;
    const int jk = blockIdx.y * blockDim.x + threadIdx.x;
    const bool active = jk < P * P;
    const int j = jk % P, k = jk / P;
    double acc[P];
#pragma unroll
    for (int i = 0; i < P; ++i) acc[i] = 0.0;
    const double4 cs = a.center_scale[e];
    for (int r = a.rng_start[e]; r < a.rng_start[e + 1]; ++r) {
        const int s0 = a.src_start[r], ns = a.src_count[r];
        for (int base = 0; base < ns; base += TS) {
            const int nt = min(TS, ns - base);
            __syncthreads();
            for (int task = threadIdx.x; task < 3 * TS; task += blockDim.x) {
                const int si = task % TS, d = task / TS;
                double* dst = d == 0 ? sx[si] : (d == 1 ? sy[si] : sz[si]);
                if (si < nt) {
                    const double4 pt = a.src[s0 + base + si];
                    const double x = (d == 0 ? pt.x - cs.x : (d == 1 ? pt.y - cs.y : pt.z - cs.z)) * cs.w;
                    const double mult = d == 2 ? pt.w : 1.0;  // fold the charge into the z factor
                    double t0 = 1.0, t1 = x;
                    dst[0] = mult;
                    if (P > 1) dst[1] = mult * x;
                    for (int n = 2; n < P; ++n) {
                        const double t2 = 2.0 * x * t1 - t0;
                        dst[n] = mult * t2;
                        t0 = t1;
                        t1 = t2;
                    }
                } else {
                    for (int n = 0; n < P; ++n) dst[n] = 0.0;
                }
            }
            __syncthreads();
            if (active) {
                for (int s = 0; s < nt; ++s) {
                    const double f = sy[s][j] * sz[s][k];
#pragma unroll
                    for (int i = 0; i < P; ++i) acc[i] = fma(f, sx[s][i], acc[i]);
                }
            }
        }
    }
    if (active) {
        double* out = a.proxy_up + (int64_t)a.slot[e] * (P * P * P) + (int64_t)P * jk;
#pragma unroll
        for (int i = 0; i < P; ++i) out[i] += acc[i];
    }
}

// Same sum for the large orders, register-tiled: a thread owns the 8 x 4
// coefficients (i in 8-block ib, j in 4-block jb) at one z-order k.  Per
// source it loads 8 x-values and 4 y-values (shared by the warp, broadcast)
// and one z-value, then does 32 multiply-adds.
template <int P>
__global__ void __launch_bounds__(128) k_c2proxy_tiled(C2ProxyArgs a) {
    constexpr int TI = 8, TJ = 4, TS = 32;
    constexpr int NIB = (P + TI - 1) / TI, NJB = (P + TJ - 1) / TJ;
    constexpr int PI = NIB * TI, PJ = NJB * TJ;  // used widths (zeros beyond P)
    // row strides: even (16-byte rows for the paired loads) and 2 mod 4
    // doubles, so the Chebyshev writes of 32 sources at one degree spread
    // over 8 bank groups instead of 2
    constexpr int LX = (PI % 4 == 2) ? PI : PI + 2, LY = (PJ % 4 == 2) ? PJ : PJ + 2;
    constexpr int NTASK = P * NJB * NIB;
    __shared__ __align__(16) double sx[TS][LX];
    __shared__ __align__(16) double sy[TS][LY];
    __shared__ double sz[TS][P | 1];
    const int e = blockIdx.x;
    const int task = blockIdx.y * blockDim.x + threadIdx.x;
    const bool active = task < NTASK;
    const int k = task % P, jb = (task / P) % NJB, ib = task / (P * NJB);
    double acc[TI][TJ];
#pragma unroll
    for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int t = 0; t < TJ; ++t) acc[i][t] = 0.0;
    const double4 cs = a.center_scale[e];
    for (int r = a.rng_start[e]; r < a.rng_start[e + 1]; ++r) {
        const int s0 = a.src_start[r], ns = a.src_count[r];
        for (int base = 0; base < ns; base += TS) {
            const int nt = min(TS, ns - base);
            __syncthreads();
            if (threadIdx.x < 3 * TS) {
                const int si = threadIdx.x % TS, d = threadIdx.x / TS;
                double* dst = d == 0 ? sx[si] : (d == 1 ? sy[si] : sz[si]);
                const int len = d == 0 ? PI : (d == 1 ? PJ : P);
                if (si < nt) {
                    const double4 pt = a.src[s0 + base + si];
                    const double x = (d == 0 ? pt.x - cs.x : (d == 1 ? pt.y - cs.y : pt.z - cs.z)) * cs.w;
                    const double mult = d == 2 ? pt.w : 1.0;  // fold the charge into the z factor
                    double t0 = 1.0, t1 = x;
                    dst[0] = mult;
                    if (P > 1) dst[1] = mult * x;
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
            if (active) {
#pragma unroll 2
                for (int s = 0; s < nt; ++s) {
                    double xv[TI], yz[TJ];
                    const double2* xr = reinterpret_cast<const double2*>(&sx[s][ib * TI]);
#pragma unroll
                    for (int i = 0; i < TI / 2; ++i) {
                        const double2 v = xr[i];
                        xv[2 * i] = v.x;
                        xv[2 * i + 1] = v.y;
                    }
                    const double z = sz[s][k];
                    const double2* yr = reinterpret_cast<const double2*>(&sy[s][jb * TJ]);
#pragma unroll
                    for (int t = 0; t < TJ / 2; ++t) {
                        const double2 v = yr[t];
                        yz[2 * t] = v.x * z;
                        yz[2 * t + 1] = v.y * z;
                    }
#pragma unroll
                    for (int i = 0; i < TI; ++i)
#pragma unroll
                        for (int t = 0; t < TJ; ++t) acc[i][t] = fma(xv[i], yz[t], acc[i][t]);
                }
            }
        }
    }
    if (!active) return;
    // a centre's moments are written here first (its children's translations
    // are added afterwards) and every coefficient by exactly one thread: store
    double* out = a.proxy_up + (int64_t)a.slot[e] * (P * P * P) + (int64_t)P * P * k;
#pragma unroll
    for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int t = 0; t < TJ; ++t) {
            const int ii = ib * TI + i, jj = jb * TJ + t;
            if (ii < P && jj < P) out[ii + P * jj] = acc[i][t];
        }
}

void launch_c2proxy(const C2ProxyArgs& a, int p, cudaStream_t s) {
    if (a.n_centers <= 0) return;
    const dim3 grid(a.n_centers, (p * p + 127) / 128);
    auto tiled_grid = [&](int q) {
        const int ntask = q * ((q + 3) / 4) * ((q + 7) / 8);
        return dim3(a.n_centers, (ntask + 127) / 128);
    };
    switch (p) {
        case 9: k_c2proxy<9><<<grid, 128, 0, s>>>(a); break;
        case 18: k_c2proxy<18><<<grid, 128, 0, s>>>(a); break;
        case 28: k_c2proxy_tiled<28><<<tiled_grid(28), 128, 0, s>>>(a); break;
        case 38: k_c2proxy_tiled<38><<<tiled_grid(38), 128, 0, s>>>(a); break;
        default: throw std::runtime_error("unsupported expansion order");
    }
}

// ============================================================================
// batched separable contraction
// ============================================================================
template <typename TO>
__device__ __forceinline__ void store_out(TO* p, double2 v, int mode, double scale);

template <>
__device__ __forceinline__ void store_out<double>(double* p, double2 v, int mode, double scale) {
    if (mode == kStore)
        *p = v.x;
    else if (mode == kAdd)
        *p += v.x;
    else
        *p += scale * v.x;
}
template <>
__device__ __forceinline__ void store_out<cd>(cd* p, double2 v, int mode, double) {
    if (mode == kStore) {
        *p = cd{v.x, v.y};
    } else {
        cd o = *p;
        *p = cd{o.x + v.x, o.y + v.y};
    }
}

// out = old + v (kAdd) or old + scale * Re v (kAddRealScaled)
template <typename TO>
__device__ __forceinline__ void store_acc(TO* p, TO old, double2 v, int mode, double scale);
template <>
__device__ __forceinline__ void store_acc<double>(double* p, double old, double2 v, int mode, double scale) {
    *p = mode == kAdd ? old + v.x : old + scale * v.x;
}
template <>
__device__ __forceinline__ void store_acc<cd>(cd* p, cd old, double2 v, int, double) {
    *p = cd{old.x + v.x, old.y + v.y};
}

// Asynchronous global -> shared copy of one 8- or 16-byte element.
template <int B>
__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem);
template <>
__device__ __forceinline__ void cp_async_elem<8>(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
                 : "memory");
}
template <>
__device__ __forceinline__ void cp_async_elem<16>(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
                 : "memory");
}

// Accumulator and multiply-add of each (input, matrix, output) type triple.
// CCR keeps only the real part, the only one it stores.  mac_re / mac_im
// multiply by a matrix entry that is real (m) or imaginary (i m).
template <typename TI, typename TM, typename TO>
struct CPol;
template <>
struct CPol<double, double, double> {
    using A = double;
    static __device__ __forceinline__ A zero() { return 0.0; }
    static __device__ __forceinline__ void mac(A& c, double m, double x) { c = fma(m, x, c); }
    static __device__ __forceinline__ double2 out(A c) { return make_double2(c, 0.0); }
};
template <>
struct CPol<double, cd, cd> {
    using A = double2;
    static __device__ __forceinline__ A zero() { return make_double2(0.0, 0.0); }
    static __device__ __forceinline__ void mac(A& c, cd m, double x) {
        c.x = fma(m.x, x, c.x);
        c.y = fma(m.y, x, c.y);
    }
    static __device__ __forceinline__ void mac_re(A& c, double m, double x) { c.x = fma(m, x, c.x); }
    static __device__ __forceinline__ void mac_im(A& c, double m, double x) { c.y = fma(m, x, c.y); }
    static __device__ __forceinline__ double2 out(A c) { return c; }
};
template <>
struct CPol<cd, cd, cd> {
    using A = double2;
    static __device__ __forceinline__ A zero() { return make_double2(0.0, 0.0); }
    static __device__ __forceinline__ void mac(A& c, cd m, cd x) {
        c.x = fma(m.x, x.x, c.x);
        c.x = fma(-m.y, x.y, c.x);
        c.y = fma(m.x, x.y, c.y);
        c.y = fma(m.y, x.x, c.y);
    }
    static __device__ __forceinline__ void mac_re(A& c, double m, cd x) {
        c.x = fma(m, x.x, c.x);
        c.y = fma(m, x.y, c.y);
    }
    static __device__ __forceinline__ void mac_im(A& c, double m, cd x) {
        c.x = fma(-m, x.y, c.x);
        c.y = fma(m, x.x, c.y);
    }
    static __device__ __forceinline__ double2 out(A c) { return c; }
};
template <>
struct CPol<cd, cd, double> {
    using A = double;
    static __device__ __forceinline__ A zero() { return 0.0; }
    static __device__ __forceinline__ void mac(A& c, cd m, cd x) {
        c = fma(m.x, x.x, c);
        c = fma(-m.y, x.y, c);
    }
    static __device__ __forceinline__ void mac_re(A& c, double m, cd x) { c = fma(m, x.x, c); }
    static __device__ __forceinline__ void mac_im(A& c, double m, cd x) { c = fma(-m, x.y, c); }
    static __device__ __forceinline__ double2 out(A c) { return make_double2(c, 0.0); }
};

// Loads TA consecutive matrix values of one row of the shared tile.
template <typename T, int TA>
__device__ __forceinline__ void load_row(T (&m)[TA], const T* row) {
    if constexpr (sizeof(T) == 8 && TA % 2 == 0) {
#pragma unroll
        for (int t = 0; t < TA; t += 2) {
            const double2 v = reinterpret_cast<const double2*>(row)[t / 2];
            m[t] = v.x;
            m[t + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int t = 0; t < TA; ++t) m[t] = row[t];
    }
}

// One CTA = one entry x a tile of RB = WR*32*TR rows; 8 warps as WA column
// groups x WR row groups.  Lane l of a warp owns rows l + 32 j (j < TR) of its
// row group; column group g owns the output columns a = k*WA*TA + g + WA*t
// (t < TA) of column chunk k, stored contiguously in the shared matrix tile.
// Per step of the contracted index a lane loads TR inputs (consecutive across
// lanes) and TA matrix values (one broadcast per pair), then does TR*TA
// multiply-adds from registers.  S selects the matrix structure used (see
// ContractStruct): the skipped entries are the rounding-level zeros of the
// triangular parent/child matrices and of the real/imaginary plane-wave tables.
template <typename TI, typename TM, typename TO, int TR, int TA, int WA, int S, bool ACC>
__device__ __forceinline__ void contract_body(const ContractArgs& a, unsigned char* smem_raw) {
    using Pol = CPol<TI, TM, TO>;
    using Acc = typename Pol::A;
    constexpr bool PAR = (S == kParIn || S == kParOut);
    using SMT = typename std::conditional<PAR, double, TM>::type;
    constexpr int WR = 8 / WA;
    constexpr int RB = WR * 32 * TR;
    constexpr int LD = RB + 1;  // odd stride: the transposing stores spread over the banks
    constexpr int CW = WA * TA;
    const int ni = a.ni, na = a.na, R = a.R;
    const int napad = (na + CW - 1) / CW * CW;
    const int e = blockIdx.x, r0 = blockIdx.y * RB;
    SMT* sM = reinterpret_cast<SMT*>(smem_raw);  // [ni][napad], permuted columns, zero beyond na
    TI* sIn = reinterpret_cast<TI*>(smem_raw + ((size_t)ni * napad * sizeof(SMT) + 15) / 16 * 16);  // [ni][LD]
    const TI* in = reinterpret_cast<const TI*>(a.in) + (a.in_off ? a.in_off[e] : (int64_t)e * a.in_stride);
    TO* out = reinterpret_cast<TO*>(a.out) + (a.out_off ? a.out_off[e] : (int64_t)e * a.out_stride);
    const TM* mat = reinterpret_cast<const TM*>(a.mat) + (a.mat_off ? a.mat_off[e] : 0);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // fill: asynchronous element copies, all in flight at once (the transpose
    // of the input tile and the column permutation of the matrix happen in
    // the copies' destination addresses)
    for (int i = w; i < ni; i += 8)
        for (int c = lane; c < napad; c += 32) {
            const int kk = c / CW, rem = c - kk * CW, g = rem / TA, t = rem - g * TA;
            const int col = kk * CW + g + WA * t;
            SMT* dst = sM + i * napad + c;
            if (col >= na) {
                *dst = SMT{};
            } else if constexpr (PAR) {
                const bool re = S == kParIn ? (i & 1) == 0 : (col & 1) == 0;
                cp_async_elem<8>(dst, reinterpret_cast<const double*>(mat + col + (int64_t)na * i) + (re ? 0 : 1));
            } else {
                cp_async_elem<sizeof(TM)>(dst, mat + col + (int64_t)na * i);
            }
        }
    const int nr = min(RB, R - r0);
    const TI* inb = in + (int64_t)ni * r0;
    for (int rr = w; rr < RB; rr += 8)
        for (int i = lane; i < ni; i += 32) {
            if (rr < nr)
                cp_async_elem<sizeof(TI)>(sIn + i * LD + rr, inb + (int64_t)rr * ni + i);
            else
                sIn[i * LD + rr] = TI{};
        }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const int wa = w % WA, wr = w / WA;
    const int rbase = wr * 32 * TR + lane;
    for (int k0 = 0; k0 < na; k0 += CW) {
        if (k0 + wa >= na) break;
        Acc acc[TR][TA];
#pragma unroll
        for (int j = 0; j < TR; ++j)
#pragma unroll
            for (int t = 0; t < TA; ++t) acc[j][t] = Pol::zero();
        const SMT* mcol = sM + k0 + wa * TA;
        if constexpr (S == kTriUpper || S == kTriLower) {
            // square matrix in one chunk (ni <= CW): the contracted indices
            // i in [WA s, WA s + WA) meet the columns a_t = wa + WA t with
            // t >= s (upper: M(a,i) = 0 for i > a) or t <= s (lower: 0 for i < a)
#pragma unroll
            for (int sg = 0; sg < TA; ++sg) {
#pragma unroll
                for (int q = 0; q < WA; ++q) {
                    const int i = WA * sg + q;
                    if (i >= ni) break;
                    TI x[TR];
#pragma unroll
                    for (int j = 0; j < TR; ++j) x[j] = sIn[i * LD + rbase + 32 * j];
                    SMT m[TA];
                    load_row<SMT, TA>(m, mcol + (size_t)i * napad);
#pragma unroll
                    for (int t = 0; t < TA; ++t) {
                        if (S == kTriUpper ? t < sg : t > sg) continue;
#pragma unroll
                        for (int j = 0; j < TR; ++j) Pol::mac(acc[j][t], m[t], x[j]);
                    }
                }
            }
        } else if constexpr (S == kParIn) {
            // entry real for even contracted index, imaginary for odd
            for (int i = 0; i < ni; ++i) {
                TI x[TR];
#pragma unroll
                for (int j = 0; j < TR; ++j) x[j] = sIn[i * LD + rbase + 32 * j];
                SMT m[TA];
                load_row<SMT, TA>(m, mcol + (size_t)i * napad);
                if ((i & 1) == 0) {
#pragma unroll
                    for (int t = 0; t < TA; ++t)
#pragma unroll
                        for (int j = 0; j < TR; ++j) Pol::mac_re(acc[j][t], m[t], x[j]);
                } else {
#pragma unroll
                    for (int t = 0; t < TA; ++t)
#pragma unroll
                        for (int j = 0; j < TR; ++j) Pol::mac_im(acc[j][t], m[t], x[j]);
                }
            }
        } else if constexpr (S == kParOut) {
            // entry real for even output column, imaginary for odd: all the
            // columns of a group share the parity of k0 + wa (WA, CW even)
            const bool re = ((k0 + wa) & 1) == 0;
            for (int i = 0; i < ni; ++i) {
                TI x[TR];
#pragma unroll
                for (int j = 0; j < TR; ++j) x[j] = sIn[i * LD + rbase + 32 * j];
                SMT m[TA];
                load_row<SMT, TA>(m, mcol + (size_t)i * napad);
                if (re) {
#pragma unroll
                    for (int t = 0; t < TA; ++t)
#pragma unroll
                        for (int j = 0; j < TR; ++j) Pol::mac_re(acc[j][t], m[t], x[j]);
                } else {
#pragma unroll
                    for (int t = 0; t < TA; ++t)
#pragma unroll
                        for (int j = 0; j < TR; ++j) Pol::mac_im(acc[j][t], m[t], x[j]);
                }
            }
        } else {
#pragma unroll 2
            for (int i = 0; i < ni; ++i) {
                TI x[TR];
#pragma unroll
                for (int j = 0; j < TR; ++j) x[j] = sIn[i * LD + rbase + 32 * j];
                SMT m[TA];
                load_row<SMT, TA>(m, mcol + (size_t)i * napad);
#pragma unroll
                for (int t = 0; t < TA; ++t)
#pragma unroll
                    for (int j = 0; j < TR; ++j) Pol::mac(acc[j][t], m[t], x[j]);
            }
        }
        if constexpr (!ACC) {
#pragma unroll
            for (int t = 0; t < TA; ++t) {
                const int col = k0 + wa + WA * t;
                if (col >= na) break;
#pragma unroll
                for (int j = 0; j < TR; ++j) {
                    const int r = rbase + 32 * j;
                    if (r < nr) store_out<TO>(out + (r0 + r) + (int64_t)R * col, Pol::out(acc[j][t]), kStore, 1.0);
                }
            }
        } else {
            // accumulate: all the old values are loaded before the first store
            TO old[TA][TR];
#pragma unroll
            for (int t = 0; t < TA; ++t)
#pragma unroll
                for (int j = 0; j < TR; ++j) {
                    const int col = k0 + wa + WA * t, r = rbase + 32 * j;
                    old[t][j] = (col < na && r < nr) ? out[(r0 + r) + (int64_t)R * col] : TO{};
                }
#pragma unroll
            for (int t = 0; t < TA; ++t) {
                const int col = k0 + wa + WA * t;
                if (col >= na) break;
#pragma unroll
                for (int j = 0; j < TR; ++j) {
                    const int r = rbase + 32 * j;
                    if (r < nr) store_acc<TO>(out + (r0 + r) + (int64_t)R * col, old[t][j], Pol::out(acc[j][t]), a.mode, a.scale);
                }
            }
        }
    }
}

template <typename TI, typename TM, typename TO, int TR, int TA, int WA, int S, bool ACC>
__global__ void __launch_bounds__(256) k_contract(ContractArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    contract_body<TI, TM, TO, TR, TA, WA, S, ACC>(a, smem_raw);
}

template <typename TI, typename TM, typename TO, int TR, int TA, int WA, int S, bool ACC>
static void launch_contract_a(const ContractArgs& a, cudaStream_t s) {
    constexpr int RB = (8 / WA) * 32 * TR;
    constexpr bool PAR = (S == kParIn || S == kParOut);
    const int napad = (a.na + WA * TA - 1) / (WA * TA) * (WA * TA);
    const size_t msz = PAR ? sizeof(double) : sizeof(TM);
    const size_t smem = ((size_t)a.ni * napad * msz + 15) / 16 * 16 + (size_t)a.ni * (RB + 1) * sizeof(TI);
    static bool configured_dev[64] = {};
    int cur_dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&cur_dev));
    bool& configured = configured_dev[cur_dev & 63];
    if (!configured) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_contract<TI, TM, TO, TR, TA, WA, S, ACC>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        configured = true;
    }
    if (smem > 200 * 1024) throw std::runtime_error("contraction tile exceeds shared memory");
    const dim3 grid(a.n_entries, (a.R + RB - 1) / RB);
    k_contract<TI, TM, TO, TR, TA, WA, S, ACC><<<grid, 256, smem, s>>>(a);
}

template <typename TI, typename TM, typename TO, int TR, int TA, int WA, int S>
static void launch_contract_s(const ContractArgs& a, cudaStream_t s) {
    if (a.mode == kStore) return launch_contract_a<TI, TM, TO, TR, TA, WA, S, false>(a, s);
    return launch_contract_a<TI, TM, TO, TR, TA, WA, S, true>(a, s);
}

// Structure dispatch: triangular only for real square matrices that fit one
// column chunk, parity only for complex matrices; anything else runs dense.
template <typename TI, typename TM, typename TO, int TR, int TA, int WA>
static void launch_contract_k(const ContractArgs& a, cudaStream_t s) {
    constexpr bool real = sizeof(TM) == sizeof(double);
    const int st = a.structure;
    if constexpr (real) {
        if ((st == kTriUpper || st == kTriLower) && a.ni == a.na && a.ni <= WA * TA) {
            if (st == kTriUpper) return launch_contract_s<TI, TM, TO, TR, TA, WA, kTriUpper>(a, s);
            return launch_contract_s<TI, TM, TO, TR, TA, WA, kTriLower>(a, s);
        }
    } else {
        if (st == kParIn) return launch_contract_s<TI, TM, TO, TR, TA, WA, kParIn>(a, s);
        if (st == kParOut) return launch_contract_s<TI, TM, TO, TR, TA, WA, kParOut>(a, s);
    }
    return launch_contract_s<TI, TM, TO, TR, TA, WA, kDense>(a, s);
}

// Column tile TA: the smallest of the instantiated widths that covers na in
// one pass of the WA column groups (the largest otherwise, looping over na).
template <typename TI, typename TM, typename TO, int TR, int WA>
static void launch_contract_t(const ContractArgs& a, cudaStream_t s) {
    switch (std::min((a.na + WA - 1) / WA, 10)) {
        case 0:
        case 1:
        case 2: return launch_contract_k<TI, TM, TO, TR, 2, WA>(a, s);
        case 3: return launch_contract_k<TI, TM, TO, TR, 3, WA>(a, s);
        case 4: return launch_contract_k<TI, TM, TO, TR, 4, WA>(a, s);
        case 5: return launch_contract_k<TI, TM, TO, TR, 5, WA>(a, s);
        case 6: return launch_contract_k<TI, TM, TO, TR, 6, WA>(a, s);
        case 7: return launch_contract_k<TI, TM, TO, TR, 7, WA>(a, s);
        case 8: return launch_contract_k<TI, TM, TO, TR, 8, WA>(a, s);
        default: return launch_contract_k<TI, TM, TO, TR, 10, WA>(a, s);
    }
}

void launch_contract(const ContractArgs& a, ContractType t, cudaStream_t s) {
    if (a.n_entries <= 0) return;
    switch (t) {
        case kRRR: launch_contract_t<double, double, double, 2, 4>(a, s); break;
        case kRCC: launch_contract_t<double, cd, cd, 2, 8>(a, s); break;
        case kCCC: launch_contract_t<cd, cd, cd, 2, 8>(a, s); break;
        case kCCR: launch_contract_t<cd, cd, double, 2, 4>(a, s); break;
    }
}

// ============================================================================
// plane-wave shift (translation x kernel FT)
// ============================================================================
__global__ void __launch_bounds__(256) k_shift(ShiftArgs a) {
    const int e = blockIdx.x;
    const int m = blockIdx.y * blockDim.x + threadIdx.x;
    if (m >= a.M) return;
    double ar = 0.0, ai = 0.0;
    for (int t = a.term_start[e]; t < a.term_start[e + 1]; ++t) {
        const cd v = a.pw_out[(int64_t)a.term_slot[t] * a.M + m];
        const double* sh = a.shift + (int64_t)a.term_stencil[t] * 2 * a.M;
        const double sr = sh[m], si = sh[a.M + m];
        ar = fma(v.x, sr, fma(-v.y, si, ar));
        ai = fma(v.x, si, fma(v.y, sr, ai));
    }
    a.pw_in[(int64_t)e * a.M + m] = cd{ar, ai};
}

void launch_shift(const ShiftArgs& a, cudaStream_t s) {
    if (a.n_entries <= 0) return;
    const dim3 grid(a.n_entries, (a.M + 255) / 256);
    k_shift<<<grid, 256, 0, s>>>(a);
}

// ============================================================================
// proxy -> leaf targets: pot_t += sum_ijk C(i,j,k) T_i(x) T_j(y) T_k(z)
// ============================================================================
template <int P>
__global__ void __launch_bounds__(128) k_eval(EvalArgs a) {
    __shared__ double slab[P * P];
    const int e = blockIdx.x;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    const double4 cs = a.center_scale[e];
    const double* C = a.proxy_down + (int64_t)a.slot[e] * (P * P * P);
    for (int base = 0; base < nt; base += blockDim.x) {
        const int t = base + threadIdx.x;
        const bool act = t < nt;
        double tx[P];
        double y = 0.0, z = 0.0;
        {
            double x = 0.0;
            if (act) {
                const double4 pt = a.trg[t0 + t];
                x = (pt.x - cs.x) * cs.w;
                y = (pt.y - cs.y) * cs.w;
                z = (pt.z - cs.z) * cs.w;
            }
            tx[0] = 1.0;
            if (P > 1) tx[1] = x;
#pragma unroll
            for (int n = 2; n < P; ++n) tx[n] = 2.0 * x * tx[n - 1] - tx[n - 2];
        }
        double acc = 0.0;
        double za = 1.0, zb = z;
        for (int k = 0; k < P; ++k) {
            __syncthreads();
            for (int idx = threadIdx.x; idx < P * P; idx += blockDim.x) slab[idx] = C[(int64_t)k * P * P + idx];
            __syncthreads();
            double ya = 1.0, yb = y, sk = 0.0;
            for (int j = 0; j < P; ++j) {
                double r = 0.0;
#pragma unroll
                for (int i = 0; i < P; ++i) r = fma(slab[i + P * j], tx[i], r);
                sk = fma(ya, r, sk);
                const double yn = 2.0 * y * yb - ya;
                ya = yb;
                yb = yn;
            }
            acc = fma(za, sk, acc);
            const double zn = 2.0 * z * zb - za;
            za = zb;
            zb = zn;
        }
        if (act) a.pot[t0 + t] += acc;
    }
}

// Large orders, register-tiled: per leaf, D[t][(j,k)] = sum_i T_i(x_t) C[i,(j,k)]
// is a small GEMM.  Warp w takes 4 targets of the 32-target pass, lane l the 4
// columns (j,k) = cbase + 4 l .. +3 of the 128-column pass: per i it loads 4
// x-values (broadcast) and 4 coefficients, then does 16 multiply-adds.  The
// y and z factors are applied per column, and the 32 lanes' partial sums of
// a target are added by a warp reduction.
template <int P>
__global__ void __launch_bounds__(256) k_eval_tiled(EvalArgs a) {
    constexpr int TT = 4, TC = 4, NW = 8;
    constexpr int TB = NW * TT;   // targets per pass
    constexpr int CB = 32 * TC;   // columns per pass
    constexpr int LDC = CB + 2;   // padded row (16-byte aligned rows, fewer bank conflicts on the fill)
    constexpr int P2 = P * P;
    extern __shared__ __align__(16) unsigned char smem_ev[];
    // two coefficient tiles [P][LDC] (the next column pass loads while this one computes)
    auto sCb = reinterpret_cast<double(*)[LDC]>(smem_ev);
    auto sX = reinterpret_cast<double(*)[TB]>(smem_ev + sizeof(double) * 2 * P * LDC);           // [P][TB]
    auto sY = reinterpret_cast<double(*)[P + 1]>(smem_ev + sizeof(double) * P * (2 * LDC + TB));  // [TB][P + 1]
    auto sZ = sY + TB;                                                                             // [TB][P + 1]
    const int e = blockIdx.x;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    const double4 cs = a.center_scale[e];
    const double* C = a.proxy_down + (int64_t)a.slot[e] * (P * P * P);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    // asynchronous fill of the column pass starting at cbase into tile buf
    auto fill = [&](int buf, int cbase) {
        const int ncol = min(CB, P2 - cbase);
        const double* Cb = C + (int64_t)P * cbase;
        double(*sC)[LDC] = sCb + buf * P;
        for (int idx = threadIdx.x; idx < P * CB; idx += blockDim.x) {
            const int c = idx / P, i = idx - c * P;
            if (c < ncol)
                cp_async_elem<8>(&sC[i][c], Cb + idx);
            else
                sC[i][c] = 0.0;
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    for (int tbase = 0; tbase < nt; tbase += TB) {
        __syncthreads();
        if (tid < TB) {
            const int t = tbase + tid;
            double x = 0.0, y = 0.0, z = 0.0;
            const bool act = t < nt;
            if (act) {
                const double4 pt = a.trg[t0 + t];
                x = (pt.x - cs.x) * cs.w;
                y = (pt.y - cs.y) * cs.w;
                z = (pt.z - cs.z) * cs.w;
            }
            double x0 = 1.0, x1 = x, y0 = 1.0, y1 = y, z0 = 1.0, z1 = z;
            const double m = act ? 1.0 : 0.0;  // inactive targets: all-zero rows
            sX[0][tid] = m;
            sY[tid][0] = 1.0;
            sZ[tid][0] = 1.0;
            if (P > 1) {
                sX[1][tid] = m * x;
                sY[tid][1] = y;
                sZ[tid][1] = z;
            }
#pragma unroll 4
            for (int n = 2; n < P; ++n) {
                const double x2 = 2.0 * x * x1 - x0, y2 = 2.0 * y * y1 - y0, z2 = 2.0 * z * z1 - z0;
                sX[n][tid] = m * x2;
                sY[tid][n] = y2;
                sZ[tid][n] = z2;
                x0 = x1;
                x1 = x2;
                y0 = y1;
                y1 = y2;
                z0 = z1;
                z1 = z2;
            }
        }
        double part[TT];
#pragma unroll
        for (int q = 0; q < TT; ++q) part[q] = 0.0;
        __syncthreads();  // previous target pass done with both tiles
        fill(0, 0);
        for (int pass = 0, cbase = 0; cbase < P2; ++pass, cbase += CB) {
            if (cbase + CB < P2) {
                fill((pass + 1) & 1, cbase + CB);
                asm volatile("cp.async.wait_group 1;" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;" ::: "memory");
            }
            __syncthreads();  // this pass's tile (and the Chebyshev rows) visible to all
            double(*sC)[LDC] = sCb + (pass & 1) * P;
            double d[TT][TC];
#pragma unroll
            for (int q = 0; q < TT; ++q)
#pragma unroll
                for (int r = 0; r < TC; ++r) d[q][r] = 0.0;
#pragma unroll 2
            for (int i = 0; i < P; ++i) {
                const double2 xa = *reinterpret_cast<const double2*>(&sX[i][w * TT]);
                const double2 xb = *reinterpret_cast<const double2*>(&sX[i][w * TT + 2]);
                const double2 ca = *reinterpret_cast<const double2*>(&sC[i][lane * TC]);
                const double2 cb = *reinterpret_cast<const double2*>(&sC[i][lane * TC + 2]);
                const double xv[TT] = {xa.x, xa.y, xb.x, xb.y};
                const double cv[TC] = {ca.x, ca.y, cb.x, cb.y};
#pragma unroll
                for (int q = 0; q < TT; ++q)
#pragma unroll
                    for (int r = 0; r < TC; ++r) d[q][r] = fma(xv[q], cv[r], d[q][r]);
            }
#pragma unroll
            for (int r = 0; r < TC; ++r) {
                const int col = cbase + lane * TC + r;
                if (col >= P2) break;
                const int j = col % P, k = col / P;
#pragma unroll
                for (int q = 0; q < TT; ++q) part[q] = fma(d[q][r], sY[w * TT + q][j] * sZ[w * TT + q][k], part[q]);
            }
            __syncthreads();  // every warp done with this tile before it is refilled
        }
#pragma unroll
        for (int q = 0; q < TT; ++q) {
            double v = part[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            const int t = tbase + w * TT + q;
            if (lane == 0 && t < nt) a.pot[t0 + t] += v;
        }
    }
}

template <int P>
static void launch_eval_tiled(const EvalArgs& a, cudaStream_t s) {
    constexpr int TB = 32, LDC = 130;
    constexpr size_t smem = sizeof(double) * ((size_t)P * (2 * LDC + TB) + 2 * (size_t)TB * (P + 1));
    static bool configured[64] = {};
    int dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_eval_tiled<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured[dev] = true;
    }
    k_eval_tiled<P><<<a.n_leaves, 256, smem, s>>>(a);
}

void launch_eval(const EvalArgs& a, int p, cudaStream_t s) {
    if (a.n_leaves <= 0) return;
    switch (p) {
        case 9: k_eval<9><<<a.n_leaves, 128, 0, s>>>(a); break;
        case 18: k_eval<18><<<a.n_leaves, 128, 0, s>>>(a); break;
        case 28: launch_eval_tiled<28>(a, s); break;
        case 38: launch_eval_tiled<38>(a, s); break;
        default: throw std::runtime_error("unsupported expansion order");
    }
}

// ============================================================================
// residual near field
// ============================================================================
template <int NC>
__global__ void __launch_bounds__(128) k_near(NearArgs a) {
    // 2 targets per thread (256 per pass); sources in chunks of 32, each chunk
    // skipped when its bounding box lies farther than b from every target of
    // the pass (the points inside a leaf follow a Morton curve, so chunks are
    // compact)
    constexpr int TPT = 2, CH = 32;
    __shared__ double4 ss[CH];
    __shared__ double sbox[4][6];
    const int e = blockIdx.x;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double c[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i) c[i] = a.coef[i];
    for (int base = 0; base < nt; base += TPT * 128) {
        double4 tp[TPT];
        double acc[TPT];
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
#pragma unroll
        for (int u = 0; u < TPT; ++u) {
            const int t = base + threadIdx.x + u * 128;
            tp[u] = t < nt ? a.trg[t0 + t] : make_double4(1e300, 1e300, 1e300, 0.0);
            acc[u] = 0.0;
            if (t < nt) {
                lo[0] = fmin(lo[0], tp[u].x); hi[0] = fmax(hi[0], tp[u].x);
                lo[1] = fmin(lo[1], tp[u].y); hi[1] = fmax(hi[1], tp[u].y);
                lo[2] = fmin(lo[2], tp[u].z); hi[2] = fmax(hi[2], tp[u].z);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
                hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
            }
        __syncthreads();
        if (lane == 0)
            for (int d = 0; d < 3; ++d) {
                sbox[warp][d] = lo[d];
                sbox[warp][3 + d] = hi[d];
            }
        __syncthreads();
        for (int d = 0; d < 3; ++d) {
            lo[d] = fmin(fmin(sbox[0][d], sbox[1][d]), fmin(sbox[2][d], sbox[3][d]));
            hi[d] = fmax(fmax(sbox[0][3 + d], sbox[1][3 + d]), fmax(sbox[2][3 + d], sbox[3][3 + d]));
        }
        for (int pr = a.pair_start[e]; pr < a.pair_start[e + 1]; ++pr) {
            const int s0 = a.pair_src_start[pr], ns = a.pair_src_count[pr];
            const double b = a.pair_bsize[pr];
            const double d2max = b * b, rsc = 2.0 / b, cen = -0.5 * b;
            const int cb = a.pair_chunk_base[pr];
            for (int sb = 0; sb < ns; sb += CH) {
                const float4 clo = __ldg(a.chunk_lo + cb + sb / CH), chi = __ldg(a.chunk_hi + cb + sb / CH);
                const double gx = fmax(0.0, fmax((double)clo.x - hi[0], lo[0] - (double)chi.x));
                const double gy = fmax(0.0, fmax((double)clo.y - hi[1], lo[1] - (double)chi.y));
                const double gz = fmax(0.0, fmax((double)clo.z - hi[2], lo[2] - (double)chi.z));
                if (fma(gx, gx, fma(gy, gy, gz * gz)) > d2max * (1.0 + 1e-12)) continue;  // uniform over the CTA
                __syncthreads();
                if ((int)threadIdx.x < CH && sb + (int)threadIdx.x < ns) ss[threadIdx.x] = a.src[s0 + sb + threadIdx.x];
                __syncthreads();
                const int m = min(CH, ns - sb);
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
                            acc[u] = fma(y.w * pv, rinv, acc[u]);
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < TPT; ++u) {
            const int t = base + threadIdx.x + u * 128;
            if (t < nt) a.pot[t0 + t] += acc[u];
        }
    }
}

void launch_near(const NearArgs& a, cudaStream_t s) {
    if (a.n_leaves <= 0) return;
    switch (a.nc) {
#define PDMK_NEAR_CASE(NC) \
    case NC: k_near<NC><<<a.n_leaves, 128, 0, s>>>(a); break;
        PDMK_NEAR_CASE(5)
        PDMK_NEAR_CASE(6)
        PDMK_NEAR_CASE(9)
        PDMK_NEAR_CASE(11)
        PDMK_NEAR_CASE(12)
        PDMK_NEAR_CASE(15)
        PDMK_NEAR_CASE(17)
        PDMK_NEAR_CASE(18)
        PDMK_NEAR_CASE(22)
        PDMK_NEAR_CASE(23)
        PDMK_NEAR_CASE(25)
#undef PDMK_NEAR_CASE
        default: throw std::runtime_error("unsupported residual polynomial length");
    }
}

// ============================================================================
// final gather
// ============================================================================
__global__ void k_finalize(const double* __restrict__ pot, const double* __restrict__ far, const double4* __restrict__ trg,
                           const int* __restrict__ perm, const double* __restrict__ q, double* __restrict__ out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int u = perm[i];
    out[u] = pot[i] + far[i] - trg[i].w * q[u];
}

void launch_finalize(const double* pot_sorted, const double* far_sorted, const double4* trg, const int* trg_perm,
                     const double* q_user, double* pot_user, int n, cudaStream_t s) {
    if (n <= 0) return;
    k_finalize<<<(n + 255) / 256, 256, 0, s>>>(pot_sorted, far_sorted, trg, trg_perm, q_user, pot_user, n);
}

// ============================================================================
// FMA throughput probe (for roofline denominators): 8 independent FMA chains
// per thread; the result is written only if it equals a sentinel that it
// cannot reach, so the chains stay live.
// ============================================================================
template <typename T>
__global__ void __launch_bounds__(256) k_fma_probe(T b, T c, int iters, T* sink) {
    T a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = (T)(threadIdx.x + i) * (T)1e-3;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = fma(a[i], b, c);
        }
    }
    T s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += a[i];
    if (s == (T)-12345.678) sink[threadIdx.x] = s;
}

double fma_probe_tflops(bool fp64) {
    int dev = 0, sms = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    PDMK_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, threads = 256, iters = fp64 ? 2000 : 8000;
    void* sink = nullptr;
    PDMK_CUDA_CHECK(cudaMalloc(&sink, 256 * sizeof(double)));
    cudaEvent_t e0, e1;
    PDMK_CUDA_CHECK(cudaEventCreate(&e0));
    PDMK_CUDA_CHECK(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        PDMK_CUDA_CHECK(cudaEventRecord(e0));
        if (fp64)
            k_fma_probe<double><<<blocks, threads>>>(0.999999, 1e-7, iters, (double*)sink);
        else
            k_fma_probe<float><<<blocks, threads>>>(0.9999f, 1e-7f, iters, (float*)sink);
        PDMK_CUDA_CHECK(cudaEventRecord(e1));
        PDMK_CUDA_CHECK(cudaEventSynchronize(e1));
        float ms = 0;
        PDMK_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0) best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    return flops / (best * 1e-3) / 1e12;
}

__global__ void k_desort_parts(const double* __restrict__ pot, const double* __restrict__ far,
                               const double4* __restrict__ trg, const int* __restrict__ perm,
                               const double* __restrict__ q, double* __restrict__ tree_part,
                               double* __restrict__ far_part, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int u = perm[i];
    tree_part[u] = pot[i] - trg[i].w * q[u];
    far_part[u] = far[i];
}

void launch_desort_parts(const double* pot_sorted, const double* far_sorted, const double4* trg, const int* trg_perm,
                         const double* q_user, double* tree_part, double* far_part, int n, cudaStream_t s) {
    if (n <= 0) return;
    k_desort_parts<<<(n + 255) / 256, 256, 0, s>>>(pot_sorted, far_sorted, trg, trg_perm, q_user, tree_part,
                                                   far_part, n);
}

// ============================================================================
// NUFFT: exponential-of-semicircle spreading kernel phi(z) = exp(beta (sqrt(1-z^2) - 1))
// (Barnett, Magland, af Klinteberg, SIAM J. Sci. Comput. 41 (2019)), width W grid cells.
// ============================================================================
__device__ __forceinline__ double es_kernel(double z, double beta) {
    const double z2 = z * z;
    return z2 < 1.0 ? exp(beta * (sqrt(1.0 - z2) - 1.0)) : 0.0;
}

__device__ __forceinline__ int wrapi(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// Spread: each CTA builds one leaf's subgrid S(i,j,k) = sum_pts q Bx_i By_j Bz_k in
// registers (thread = (j,k) column, x along the register array) and flushes it
// once into the global periodic grid with atomics.
template <int W, int NX>
__global__ void __launch_bounds__(128) k_spread(NufftArgs a) {
    constexpr int TS = 32;
    __shared__ double sBx[TS][NX];
    __shared__ double sKy[TS][W], sKz[TS][W];
    __shared__ int sBy[TS], sBz[TS];
    __shared__ double sQ[TS];
    const int e = blockIdx.x;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    const int4 org = a.sub_origin[e], ext = a.sub_extent[e];
    const double* __restrict__ qs = a.q_sorted + blockIdx.z * a.rhs_q_stride;
    double* __restrict__ grid = a.grid + blockIdx.z * a.rhs_grid_stride;
    const int jk = blockIdx.y * blockDim.x + threadIdx.x;
    const bool active = jk < ext.y * ext.z;
    const int kk = jk % max(ext.z, 1), jj = jk / max(ext.z, 1);
    const double hw = 0.5 * W;
    double acc[NX];
#pragma unroll
    for (int i = 0; i < NX; ++i) acc[i] = 0.0;
    for (int base = 0; base < nt; base += TS) {
        const int m = min(TS, nt - base);
        __syncthreads();
        if (threadIdx.x < TS) {
            const int s = threadIdx.x;
            if (s < m) {
                const double4 t = a.pt_t[t0 + base + s];
                const int4 l0 = a.pt_l0[t0 + base + s];
                const int bx = l0.x - org.x;
                for (int i = 0; i < NX; ++i) {
                    const int o = i - bx;
                    sBx[s][i] = (o >= 0 && o < W) ? es_kernel((t.x - (double)(l0.x + o)) / hw, a.es_beta) : 0.0;
                }
                for (int c = 0; c < W; ++c) {
                    sKy[s][c] = es_kernel((t.y - (double)(l0.y + c)) / hw, a.es_beta);
                    sKz[s][c] = es_kernel((t.z - (double)(l0.z + c)) / hw, a.es_beta);
                }
                sBy[s] = l0.y - org.y;
                sBz[s] = l0.z - org.z;
                sQ[s] = qs[t0 + base + s];
            }
        }
        __syncthreads();
        if (active) {
            for (int s = 0; s < m; ++s) {
                const int dj = jj - sBy[s], dk = kk - sBz[s];
                if (dj < 0 || dj >= W || dk < 0 || dk >= W) continue;
                const double f = sQ[s] * sKy[s][dj] * sKz[s][dk];
#pragma unroll
                for (int i = 0; i < NX; ++i) acc[i] = fma(f, sBx[s][i], acc[i]);
            }
        }
    }
    if (!active) return;
    const int gy = wrapi(org.y + jj, a.n2), gz = wrapi(org.z + kk, a.n3);
#pragma unroll
    for (int i = 0; i < NX; ++i) {
        if (i < ext.x && acc[i] != 0.0) {
            const int gx = wrapi(org.x + i, a.n1);
            atomicAdd(grid + ((int64_t)gx * a.n2 + gy) * a.n3 + gz, acc[i]);
        }
    }
}

template <int W>
__global__ void __launch_bounds__(128) k_interp(NufftArgs a) {
    const int e = blockIdx.x;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    const double hw = 0.5 * W;
    const double* __restrict__ grid = a.grid + blockIdx.z * a.rhs_grid_stride;
    double* __restrict__ far = a.far + blockIdx.z * a.rhs_far_stride;
    for (int tl = threadIdx.x; tl < nt; tl += blockDim.x) {
        const int t = (a.interp_order ? a.interp_order[t0 + tl] : t0 + tl) - t0;
        const double4 tt = a.pt_t[t0 + t];
        const int4 l0 = a.pt_l0[t0 + t];
        double kx[W], ky[W], kz[W];
        int iy[W], iz[W];
#pragma unroll
        for (int c = 0; c < W; ++c) {
            kx[c] = es_kernel((tt.x - (double)(l0.x + c)) / hw, a.es_beta);
            ky[c] = es_kernel((tt.y - (double)(l0.y + c)) / hw, a.es_beta);
            kz[c] = es_kernel((tt.z - (double)(l0.z + c)) / hw, a.es_beta);
            iy[c] = wrapi(l0.y + c, a.n2);
            iz[c] = wrapi(l0.z + c, a.n3);
        }
        double u = 0.0;
#pragma unroll 1
        for (int ia = 0; ia < W; ++ia) {
            const double* gx = grid + (int64_t)wrapi(l0.x + ia, a.n1) * a.n2 * a.n3;
            double sa = 0.0;
#pragma unroll
            for (int ib = 0; ib < W; ++ib) {
                const double* gy = gx + (int64_t)iy[ib] * a.n3;
                double sb = 0.0;
#pragma unroll
                for (int ic = 0; ic < W; ++ic) sb = fma(kz[ic], __ldg(gy + iz[ic]), sb);
                sa = fma(ky[ib], sb, sa);
            }
            u = fma(kx[ia], sa, u);
        }
        far[t0 + t] = u;
    }
}

__global__ void k_multiply(cd* spec, const double* mult, int64_t n, int64_t total) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const double m = mult[i % n];
    cd v = spec[i];
    spec[i] = cd{v.x * m, v.y * m};
}

void launch_multiply(cd* spec, const double* mult, int64_t n, cudaStream_t s, int nrhs) {
    if (n <= 0 || nrhs <= 0) return;
    const int64_t total = n * nrhs;
    k_multiply<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(spec, mult, n, total);
}

template <int W>
static void launch_spread_w(const NufftArgs& a, int max_jk, int max_ex, cudaStream_t s, int nrhs) {
    const dim3 grid(a.n_leaves, (max_jk + 127) / 128, nrhs);
    if (max_ex <= 16)
        k_spread<W, 16><<<grid, 128, 0, s>>>(a);
    else if (max_ex <= 32)
        k_spread<W, 32><<<grid, 128, 0, s>>>(a);
    else if (max_ex <= 48)
        k_spread<W, 48><<<grid, 128, 0, s>>>(a);
    else
        throw std::runtime_error("NUFFT leaf subgrid too large");
}

void launch_spread(const NufftArgs& a, int max_jk, int max_ex, cudaStream_t s, int nrhs) {
    if (a.n_leaves <= 0 || nrhs <= 0) return;
    switch (a.w) {
#define PDMK_W_CASE(W) \
    case W: launch_spread_w<W>(a, max_jk, max_ex, s, nrhs); break;
        PDMK_W_CASE(4) PDMK_W_CASE(5) PDMK_W_CASE(6) PDMK_W_CASE(7) PDMK_W_CASE(8) PDMK_W_CASE(9)
        PDMK_W_CASE(10) PDMK_W_CASE(11) PDMK_W_CASE(12) PDMK_W_CASE(13) PDMK_W_CASE(14)
#undef PDMK_W_CASE
        default: throw std::runtime_error("unsupported NUFFT kernel width");
    }
}

void launch_interp(const NufftArgs& a, cudaStream_t s, int nrhs) {
    if (a.n_leaves <= 0 || nrhs <= 0) return;
    const dim3 grid(a.n_leaves, 1, nrhs);
    switch (a.w) {
#define PDMK_W_CASE(W) \
    case W: k_interp<W><<<grid, 128, 0, s>>>(a); break;
        PDMK_W_CASE(4) PDMK_W_CASE(5) PDMK_W_CASE(6) PDMK_W_CASE(7) PDMK_W_CASE(8) PDMK_W_CASE(9)
        PDMK_W_CASE(10) PDMK_W_CASE(11) PDMK_W_CASE(12) PDMK_W_CASE(13) PDMK_W_CASE(14)
#undef PDMK_W_CASE
        default: throw std::runtime_error("unsupported NUFFT kernel width");
    }
}

}  // namespace dev
}  // namespace pdmkb
