// Fused plane-wave transforms of the multi-RHS path: one CTA per (box, RHS)
// entry runs all three separable steps with the intermediate tensors in shared
// memory (the step-by-step form writes each intermediate to global memory).
//
// Outgoing (proxy -> plane wave, reference proxy.cpp:42-90):
//   pw(a,b,c) = sum_{ijk} Pxy(a,i) Pxy(b,j) Pz(c,k) proxy(i,j,k)
//   Pxy = poly2pw (n x p), Pz = poly2pw_half (n2 x p); the z axis is contracted
//   first (n2 < n keeps the intermediates smallest).
// Incoming (plane wave -> proxy, reference planewave.cpp:49-105):
//   proxy(i,j,k) += 2 Re sum_{abc} Uxy(i,a) Uxy(j,b) Uz(k,c) pw(a,b,c)
//   Uxy = pw2polyT (p x n), Uz = pw2polyTw (p x n2, half-space weights folded).
// Tensors are stored x fastest: element (i0,i1,i2) of extents (S0,S1,S2) at
// i0 + S0*(i1 + S1*i2).  Matrices are column-major (rows = output index).
#include <stdexcept>

#include "pw_fused.cuh"

namespace pdmkb {
namespace dev {

namespace {

struct cfx {
    float x, y;
};

template <typename T>
struct CplxOf;
template <>
struct CplxOf<float> {
    using type = cfx;
};
template <>
struct CplxOf<double> {
    using type = cd;
};

template <typename C, typename R>
__device__ __forceinline__ C cmac(C m, R x, C acc) {  // complex matrix x real data
    acc.x = fma(m.x, x, acc.x);
    acc.y = fma(m.y, x, acc.y);
    return acc;
}
template <typename C>
__device__ __forceinline__ C cmacc(C m, C x, C acc) {  // complex x complex
    acc.x = fma(m.x, x.x, fma(-m.y, x.y, acc.x));
    acc.y = fma(m.x, x.y, fma(m.y, x.x, acc.y));
    return acc;
}

// One separable step: dst = src with axis AX (extent SA) contracted against
// M (NA x SA, column-major), the new index at the same axis position.
// Tasks (a, u) with a the output index of the contracted axis (fastest across
// threads, so every src read is a broadcast) and u the first other axis; each
// task loops over the second other axis v.  OUT: 0 store complex, 1 store
// real part x scale.
template <int S0, int S1, int S2, int AX, int NA, int OUT, bool REAL_IN, typename C, typename R, typename TS,
          typename TD>
__device__ __forceinline__ void sep_step(const TS* __restrict__ src, TD* __restrict__ dst, const C* __restrict__ M,
                                         R scale) {
    constexpr int SA = AX == 0 ? S0 : (AX == 1 ? S1 : S2);
    constexpr int UAX = AX == 0 ? 1 : 0;
    constexpr int VAX = AX == 2 ? 1 : 2;
    constexpr int SU = UAX == 0 ? S0 : S1;
    constexpr int SV = VAX == 1 ? S1 : S2;
    constexpr int ST0 = 1, ST1 = S0, ST2 = S0 * S1;
    constexpr int sA = AX == 0 ? ST0 : (AX == 1 ? ST1 : ST2);
    constexpr int sU = UAX == 0 ? ST0 : ST1;
    constexpr int sV = VAX == 1 ? ST1 : ST2;
    constexpr int D0 = AX == 0 ? NA : S0, D1 = AX == 1 ? NA : S1;
    constexpr int DT0 = 1, DT1 = D0, DT2 = D0 * D1;
    constexpr int dA = AX == 0 ? DT0 : (AX == 1 ? DT1 : DT2);
    constexpr int dU = UAX == 0 ? DT0 : DT1;
    constexpr int dV = VAX == 1 ? DT1 : DT2;
    for (int task = threadIdx.x; task < NA * SU; task += blockDim.x) {
        const int a = task % NA, u = task / NA;
        C row[SA];
#pragma unroll
        for (int i = 0; i < SA; ++i) row[i] = M[a + NA * i];
        const TS* s0 = src + u * sU;
        TD* d0 = dst + a * dA + u * dU;
#pragma unroll 2
        for (int v = 0; v < SV; ++v) {
            C acc;
            acc.x = R(0);
            acc.y = R(0);
            const TS* sp = s0 + v * sV;
#pragma unroll
            for (int i = 0; i < SA; ++i) {
                if constexpr (REAL_IN)
                    acc = cmac(row[i], sp[i * sA], acc);
                else
                    acc = cmacc(row[i], sp[i * sA], acc);
            }
            if constexpr (OUT == 0)
                d0[v * dV] = acc;
            else
                d0[v * dV] = scale * acc.x;
        }
    }
}

template <typename T, int P, int N, int N2>
struct PwShape {
    using C = typename CplxOf<T>::type;
    // outgoing: A holds proxy (real) then (p, n, n2); B holds (p, p, n2)
    static constexpr size_t OUT_A = sizeof(C) * P * N * N2 > sizeof(T) * P * P * P ? sizeof(C) * P * N * N2
                                                                                     : sizeof(T) * P * P * P;
    static constexpr size_t OUT_B = sizeof(C) * P * P * N2;
    static constexpr size_t OUT_SMEM = OUT_A + OUT_B;
    // incoming: A holds (p, n, n2) then the real (p, p, p) result; B holds (p, p, n2)
    static constexpr size_t IN_A = sizeof(C) * P * N * N2;
    static constexpr size_t IN_B = sizeof(C) * P * P * N2;
    static constexpr size_t IN_SMEM = IN_A + IN_B;
    // staged incoming: R1 holds the input (n, n, n2), then (p, p, n2); R2 holds
    // (p, n, n2), then the real (p, p, p) result
    static constexpr size_t IN_R1 = sizeof(C) * N * N * N2;
    static constexpr size_t IN_STAGED_SMEM = IN_R1 + IN_A;
    static constexpr bool IN_STAGED = IN_STAGED_SMEM <= 227 * 1024;
};

template <typename T, int P, int N, int N2>
__global__ void __launch_bounds__(256) k_pw_out_fused(PwFused a) {
    using C = typename CplxOf<T>::type;
    using S = PwShape<T, P, N, N2>;
    extern __shared__ __align__(16) unsigned char smem_pw[];
    unsigned char* bufA = smem_pw;
    unsigned char* bufB = smem_pw + S::OUT_A;
    const int64_t ge = a.e0 + blockIdx.x;
    const int rhs = a.rhs > 0 ? a.rhs : 1;
    const int64_t eb = ge / rhs, ec = ge % rhs;
    const T* in = reinterpret_cast<const T*>(a.in) + a.in_off[eb] * rhs + ec * (int64_t)(P * P * P);
    C* out = reinterpret_cast<C*>(a.out) + a.out_off[eb] * rhs + ec * (int64_t)(N * N * N2);
    const C* Mxy = reinterpret_cast<const C*>(a.mat_a);
    const C* Mz = reinterpret_cast<const C*>(a.mat_b);
    T* pin = reinterpret_cast<T*>(bufA);
    for (int i = threadIdx.x; i < P * P * P; i += blockDim.x) pin[i] = in[i];
    __syncthreads();
    // (p,p,p) real -> (p,p,n2): contract z
    sep_step<P, P, P, 2, N2, 0, true, C, T>(pin, reinterpret_cast<C*>(bufB), Mz, T(1));
    __syncthreads();
    // (p,p,n2) -> (p,n,n2): contract y
    sep_step<P, P, N2, 1, N, 0, false, C, T>(reinterpret_cast<const C*>(bufB), reinterpret_cast<C*>(bufA), Mxy, T(1));
    __syncthreads();
    // (p,n,n2) -> (n,n,n2): contract x, straight to global (coalesced along a)
    sep_step<P, N, N2, 0, N, 0, false, C, T>(reinterpret_cast<const C*>(bufA), out, Mxy, T(1));
}

template <typename T, int P, int N, int N2>
__global__ void __launch_bounds__(512) k_pw_in_fused(PwFused a) {
    using C = typename CplxOf<T>::type;
    using S = PwShape<T, P, N, N2>;
    extern __shared__ __align__(16) unsigned char smem_pw[];
    unsigned char* bufA = smem_pw;
    unsigned char* bufB = smem_pw + S::IN_A;
    const int64_t ge = a.e0 + blockIdx.x;
    const int rhs = a.rhs > 0 ? a.rhs : 1;
    const int64_t eb = ge / rhs, ec = ge % rhs;
    const C* in = reinterpret_cast<const C*>(a.in) + (int64_t)blockIdx.x * a.in_stride;
    T* out = reinterpret_cast<T*>(a.out) + a.out_off[eb] * rhs + ec * (int64_t)(P * P * P);
    const C* Uxy = reinterpret_cast<const C*>(a.mat_a);
    const C* Uz = reinterpret_cast<const C*>(a.mat_b);
    if constexpr (S::IN_STAGED) {
        // stage the input: every element of it is read by all the tasks of one output row
        unsigned char* r1 = smem_pw;
        unsigned char* r2 = smem_pw + S::IN_R1;
        C* s1 = reinterpret_cast<C*>(r1);  // element copies: entries need not be 16-byte aligned
        for (int i = threadIdx.x; i < N * N * N2; i += blockDim.x) s1[i] = in[i];
        __syncthreads();
        sep_step<N, N, N2, 0, P, 0, false, C, T>(reinterpret_cast<const C*>(r1), reinterpret_cast<C*>(r2), Uxy, T(1));
        __syncthreads();
        sep_step<P, N, N2, 1, P, 0, false, C, T>(reinterpret_cast<const C*>(r2), reinterpret_cast<C*>(r1), Uxy, T(1));
        __syncthreads();
        T* res = reinterpret_cast<T*>(r2);
        sep_step<P, P, N2, 2, P, 1, false, C, T>(reinterpret_cast<const C*>(r1), res, Uz, T(2));
        __syncthreads();
        for (int i = threadIdx.x; i < P * P * P; i += blockDim.x) out[i] += res[i];
        return;
    }
    // (n,n,n2) from global -> (p,n,n2): contract x
    sep_step<N, N, N2, 0, P, 0, false, C, T>(in, reinterpret_cast<C*>(bufA), Uxy, T(1));
    __syncthreads();
    // (p,n,n2) -> (p,p,n2): contract y
    sep_step<P, N, N2, 1, P, 0, false, C, T>(reinterpret_cast<const C*>(bufA), reinterpret_cast<C*>(bufB), Uxy, T(1));
    __syncthreads();
    // (p,p,n2) -> (p,p,p) real, 2 Re(.): contract z into shared memory
    T* res = reinterpret_cast<T*>(bufA);
    sep_step<P, P, N2, 2, P, 1, false, C, T>(reinterpret_cast<const C*>(bufB), res, Uz, T(2));
    __syncthreads();
    for (int i = threadIdx.x; i < P * P * P; i += blockDim.x) out[i] += res[i];
}

template <typename T, int P, int N, int N2>
void launch_out_pnn(const PwFused& a, int n_entries, cudaStream_t s) {
    using S = PwShape<T, P, N, N2>;
    static bool configured[64] = {};
    int dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw std::runtime_error("device index out of range");
    if (!configured[dev]) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_pw_out_fused<T, P, N, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)S::OUT_SMEM));
        configured[dev] = true;
    }
    k_pw_out_fused<T, P, N, N2><<<n_entries, 256, S::OUT_SMEM, s>>>(a);
}

template <typename T, int P, int N, int N2>
void launch_in_pnn(const PwFused& a, int n_entries, cudaStream_t s) {
    using S = PwShape<T, P, N, N2>;
    static bool configured[64] = {};
    int dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw std::runtime_error("device index out of range");
    constexpr size_t smem = S::IN_STAGED ? S::IN_STAGED_SMEM : S::IN_SMEM;
    if (!configured[dev]) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_pw_in_fused<T, P, N, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem));
        configured[dev] = true;
    }
    k_pw_in_fused<T, P, N, N2><<<n_entries, S::IN_STAGED ? 512 : 256, smem, s>>>(a);
}

constexpr size_t kMaxSmem = 227 * 1024;

}  // namespace

template <typename T>
bool pw_fused_supported(int p, int n, int n2) {
    if (p == 9 && n == 13 && n2 == 7) return true;
    if (p == 18 && n == 27 && n2 == 14)
        return PwShape<T, 18, 27, 14>::OUT_SMEM <= kMaxSmem && PwShape<T, 18, 27, 14>::IN_SMEM <= kMaxSmem;
    return false;
}

template <typename T>
void launch_pw_out_fused(const PwFused& a, int p, int n, int n2, int n_entries, cudaStream_t s) {
    if (n_entries <= 0) return;
    if (p == 9 && n == 13 && n2 == 7)
        launch_out_pnn<T, 9, 13, 7>(a, n_entries, s);
    else if (p == 18 && n == 27 && n2 == 14)
        launch_out_pnn<T, 18, 27, 14>(a, n_entries, s);
    else
        throw std::runtime_error("fused plane-wave transform: unsupported (p, n)");
}

template <typename T>
void launch_pw_in_fused(const PwFused& a, int p, int n, int n2, int n_entries, cudaStream_t s) {
    if (n_entries <= 0) return;
    if (p == 9 && n == 13 && n2 == 7)
        launch_in_pnn<T, 9, 13, 7>(a, n_entries, s);
    else if (p == 18 && n == 27 && n2 == 14)
        launch_in_pnn<T, 18, 27, 14>(a, n_entries, s);
    else
        throw std::runtime_error("fused plane-wave transform: unsupported (p, n)");
}

template bool pw_fused_supported<float>(int, int, int);
template bool pw_fused_supported<double>(int, int, int);
template void launch_pw_out_fused<float>(const PwFused&, int, int, int, int, cudaStream_t);
template void launch_pw_out_fused<double>(const PwFused&, int, int, int, int, cudaStream_t);
template void launch_pw_in_fused<float>(const PwFused&, int, int, int, int, cudaStream_t);
template void launch_pw_in_fused<double>(const PwFused&, int, int, int, int, cudaStream_t);

}  // namespace dev
}  // namespace pdmkb
