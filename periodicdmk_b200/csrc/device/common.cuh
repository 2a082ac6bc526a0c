// Shared device helpers for the periodic DMK evaluate kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#define PDMK_CUDA_CHECK(expr)                                                                              \
    do {                                                                                                   \
        cudaError_t _e = (expr);                                                                           \
        if (_e != cudaSuccess)                                                                             \
            throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(_e) + " at " __FILE__ \
                                     ":" + std::to_string(__LINE__));                                      \
    } while (0)

namespace pdmkb {
namespace dev {

struct cd {  // complex double, 16-byte aligned
    double x, y;
};
static_assert(sizeof(cd) == 16, "cd");

__host__ __device__ __forceinline__ cd cmul(cd a, cd b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__host__ __device__ __forceinline__ cd cfma(cd a, cd b, cd c) {
    return {fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y))};
}
__host__ __device__ __forceinline__ cd cfma(double a, cd b, cd c) { return {fma(a, b.x, c.x), fma(a, b.y, c.y)}; }
__host__ __device__ __forceinline__ cd cfma(cd a, double b, cd c) { return {fma(a.x, b, c.x), fma(a.y, b, c.y)}; }
__host__ __device__ __forceinline__ double dfma(double a, double b, double c) { return fma(a, b, c); }

#ifdef __CUDACC__
template <typename T>
__device__ __forceinline__ T zero();
template <>
__device__ __forceinline__ double zero<double>() { return 0.0; }
template <>
__device__ __forceinline__ cd zero<cd>() { return {0.0, 0.0}; }

// Multiply-accumulate with mixed real/complex operands: acc += m * x.
__device__ __forceinline__ double mac(double m, double x, double acc) { return fma(m, x, acc); }
__device__ __forceinline__ cd mac(cd m, double x, cd acc) { return cfma(m, x, acc); }
__device__ __forceinline__ cd mac(double m, cd x, cd acc) { return cfma(m, x, acc); }
__device__ __forceinline__ cd mac(cd m, cd x, cd acc) { return cfma(m, x, acc); }

// 1/sqrt(x) in FP64: FP32 hardware estimate refined by two Newton steps
// y <- y (3 - x y^2) / 2 (quadratic convergence, ~2^-22 -> full precision).
__device__ __forceinline__ double rsqrt_nr(double x) {
    double y = (double)rsqrtf((float)x);
    const double h = 0.5 * x;
    y = y * fma(-h, y * y, 1.5);
    y = y * fma(-h, y * y, 1.5);
    return y;
}
#endif  // __CUDACC__

}  // namespace dev
}  // namespace pdmkb
