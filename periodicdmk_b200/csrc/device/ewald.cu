// Ewald summation on the GPU (pdmk_ewald_nufft; the reference's ewald_nufft,
// cpp/src/ewald_nufft.cpp:445-654, behind cpp/src/pdmk_capi.cpp:88-106).
//
// u_i = sum_j q_j sum_R' erfc(a r)/r  +  sum_{K != 0, |K| <= kmax} w(K) Re(S(K) e^{i K.x_i})  -  2 a / sqrt(pi) q_i,
// w(K) = 4 pi / V e^{-K^2 / 4a^2} / K^2, S(K) = sum_j q_j e^{-i K.x_j},
// E = 1/2 sum_i q_i u_i - pi Q^2 / (2 V a^2), with the reference's parameter
// choice: a = max((N pi^3 / V^2)^(1/6), s (4 pi rho / (3 n_nbr))^(1/3)),
// n_nbr = 5000 (DMK_EWALD_TARGET_NBR overrides it, as in the reference),
// r_cut = s / a, kmax = 2 s a, modes |m_d| <= ceil(kmax |a_d| / 2 pi).
//
//   * real space: the points are binned on fractional coordinates into
//     m_d = max(1, floor(h_d / r_cut)) slabs per axis (h_d the distance between
//     lattice planes), so every pair within r_cut lies within R_d =
//     ceil(r_cut m_d / h_d) bins along axis d; one CTA per target bin stages
//     the sources of each neighbour bin (with its lattice image shift) in
//     shared memory, one thread per target;
//   * reciprocal space: a type-1 / type-2 NUFFT pair with an exponential-of-
//     semicircle kernel of width 13 (tolerance 1e-12, the reference's
//     nufft_tol), upsampling 2: spreading by FP64 atomics, cuFFT D2Z, the
//     weight times the kernel deconvolution on the half spectrum, cuFFT Z2D,
//     interpolation.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../host/pswf.hpp"
#include "common.cuh"
#include "ewald.cuh"

namespace pdmkb {

namespace dev {
namespace {

constexpr int kEsW = 13;  // kernel width (points per axis)
constexpr int kRealThreads = 128;

struct RealArgs {
    const double4* pts;     // sorted by bin: x, y, z (wrapped into the cell), q
    const int* bin_start;   // nbins + 1
    int m0, m1, m2, r0, r1, r2;
    double a[9];            // lattice vectors a_d = (a[3d], a[3d+1], a[3d+2])
    double alpha, rc2;
    double* out;            // per sorted point
};

__global__ void __launch_bounds__(kRealThreads) k_ewald_real(RealArgs A) {
    __shared__ double4 sh[kRealThreads];
    const int b = blockIdx.x;
    const int i2 = b % A.m2, i1 = (b / A.m2) % A.m1, i0 = b / (A.m1 * A.m2);
    const int t0 = A.bin_start[b], t1 = A.bin_start[b + 1];
    for (int tb = t0 + (int)blockIdx.y * kRealThreads; tb < t1; tb += (int)gridDim.y * kRealThreads) {
        const int t = tb + threadIdx.x;
        const bool act = t < t1;
        const double4 p = act ? A.pts[t] : make_double4(0, 0, 0, 0);
        double acc = 0.0;
        for (int d0 = -A.r0; d0 <= A.r0; ++d0)
            for (int d1 = -A.r1; d1 <= A.r1; ++d1)
                for (int d2 = -A.r2; d2 <= A.r2; ++d2) {
                    const int j0 = i0 + d0, j1 = i1 + d1, j2 = i2 + d2;
                    const int w0 = ((j0 % A.m0) + A.m0) % A.m0, w1 = ((j1 % A.m1) + A.m1) % A.m1,
                              w2 = ((j2 % A.m2) + A.m2) % A.m2;
                    const int n0 = (j0 - w0) / A.m0, n1 = (j1 - w1) / A.m1, n2 = (j2 - w2) / A.m2;
                    // target minus the image shift, so that dx = x_t - (x_s + shift)
                    const double sx = p.x - (n0 * A.a[0] + n1 * A.a[3] + n2 * A.a[6]);
                    const double sy = p.y - (n0 * A.a[1] + n1 * A.a[4] + n2 * A.a[7]);
                    const double sz = p.z - (n0 * A.a[2] + n1 * A.a[5] + n2 * A.a[8]);
                    const int nb = (w0 * A.m1 + w1) * A.m2 + w2;
                    const int s0 = A.bin_start[nb], s1 = A.bin_start[nb + 1];
                    for (int c = s0; c < s1; c += kRealThreads) {
                        const int nc = min(kRealThreads, s1 - c);
                        __syncthreads();
                        if ((int)threadIdx.x < nc) sh[threadIdx.x] = A.pts[c + threadIdx.x];
                        __syncthreads();
                        if (!act) continue;
                        for (int k = 0; k < nc; ++k) {
                            const double4 s = sh[k];
                            const double dx = sx - s.x, dy = sy - s.y, dz = sz - s.z;
                            const double r2 = dx * dx + dy * dy + dz * dz;
                            if (r2 <= A.rc2 && r2 > 0.0) {
                                const double r = sqrt(r2);
                                acc += s.w * erfc(A.alpha * r) / r;
                            }
                        }
                    }
                }
        if (act) A.out[t] = acc;
    }
}

struct NufftE {
    const double4* pts;  // x, y, z, q (any order)
    double ainv[9];      // fractional s_d = sum_e ainv[3 d + e] x_e
    int n[3];
    double beta;         // kernel exp(beta (sqrt(1 - z^2) - 1))
    double* grid;        // n0 x n1 x n2, n2 fastest
    double* out;
    int64_t npts;
};

// kernel weights of one axis: points g0 .. g0 + W - 1
__device__ __forceinline__ int es_weights(double s, int n, double beta, double* w) {
    double u = s - floor(s);  // fractional coordinate in [0, 1)
    const double x = u * n;   // grid units
    const int g0 = (int)ceil(x - 0.5 * kEsW);
    const double inv = 2.0 / kEsW;
#pragma unroll
    for (int k = 0; k < kEsW; ++k) {
        const double z = (x - (double)(g0 + k)) * inv;
        const double t = 1.0 - z * z;
        w[k] = t > 0.0 ? exp(beta * (sqrt(t) - 1.0)) : 0.0;
    }
    return g0;
}

__device__ __forceinline__ void frac(const NufftE& a, const double4& p, double* s) {
    for (int d = 0; d < 3; ++d) s[d] = a.ainv[3 * d] * p.x + a.ainv[3 * d + 1] * p.y + a.ainv[3 * d + 2] * p.z;
}

__global__ void k_ewald_spread(NufftE a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.npts) return;
    const double4 p = a.pts[i];
    double s[3], w0[kEsW], w1[kEsW], w2[kEsW];
    frac(a, p, s);
    const int g0 = es_weights(s[0], a.n[0], a.beta, w0);
    const int g1 = es_weights(s[1], a.n[1], a.beta, w1);
    const int g2 = es_weights(s[2], a.n[2], a.beta, w2);
    for (int k0 = 0; k0 < kEsW; ++k0) {
        const int x0 = ((g0 + k0) % a.n[0] + a.n[0]) % a.n[0];
        const double q0 = p.w * w0[k0];
        for (int k1 = 0; k1 < kEsW; ++k1) {
            const int x1 = ((g1 + k1) % a.n[1] + a.n[1]) % a.n[1];
            const double q01 = q0 * w1[k1];
            double* row = a.grid + ((int64_t)x0 * a.n[1] + x1) * a.n[2];
            for (int k2 = 0; k2 < kEsW; ++k2) {
                const int x2 = ((g2 + k2) % a.n[2] + a.n[2]) % a.n[2];
                atomicAdd(row + x2, q01 * w2[k2]);
            }
        }
    }
}

__global__ void k_ewald_interp(NufftE a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.npts) return;
    const double4 p = a.pts[i];
    double s[3], w0[kEsW], w1[kEsW], w2[kEsW];
    frac(a, p, s);
    const int g0 = es_weights(s[0], a.n[0], a.beta, w0);
    const int g1 = es_weights(s[1], a.n[1], a.beta, w1);
    const int g2 = es_weights(s[2], a.n[2], a.beta, w2);
    double acc = 0.0;
    for (int k0 = 0; k0 < kEsW; ++k0) {
        const int x0 = ((g0 + k0) % a.n[0] + a.n[0]) % a.n[0];
        double a1 = 0.0;
        for (int k1 = 0; k1 < kEsW; ++k1) {
            const int x1 = ((g1 + k1) % a.n[1] + a.n[1]) % a.n[1];
            const double* row = a.grid + ((int64_t)x0 * a.n[1] + x1) * a.n[2];
            double a2 = 0.0;
            for (int k2 = 0; k2 < kEsW; ++k2) {
                const int x2 = ((g2 + k2) % a.n[2] + a.n[2]) % a.n[2];
                a2 += w2[k2] * row[x2];
            }
            a1 += w1[k1] * a2;
        }
        acc += w0[k0] * a1;
    }
    a.out[i] = acc;
}

__global__ void k_ewald_scale(cd* spec, const double* mult, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double m = mult[i];
    spec[i].x *= m;
    spec[i].y *= m;
}

int smooth_size(int lo) {
    for (int n = std::max(lo, 2);; ++n) {
        if (n % 2) continue;
        int r = n;
        for (int f : {2, 3, 5, 7})
            while (r % f == 0) r /= f;
        if (r == 1) return n;
    }
}

template <typename T>
struct DevBuf {
    T* p = nullptr;
    explicit DevBuf(size_t n) { PDMK_CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T))); }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

struct FftPlan {
    cufftHandle h = 0;
    ~FftPlan() {
        if (h) cufftDestroy(h);
    }
};

}  // namespace
}  // namespace dev

void ewald_gpu(const double* cell, int n, const double* pos, const double* q, double s, double* pot, double* energy,
               EwaldInfo* info) {
    using namespace dev;
    if (n <= 0) throw std::invalid_argument("N must be positive");
    if (!(s > 0) || !std::isfinite(s)) throw std::invalid_argument("s must be positive");
    const double* a[3] = {cell, cell + 3, cell + 6};
    auto cross = [](const double* u, const double* v, double* w) {
        w[0] = u[1] * v[2] - u[2] * v[1];
        w[1] = u[2] * v[0] - u[0] * v[2];
        w[2] = u[0] * v[1] - u[1] * v[0];
    };
    auto dot = [](const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
    double c[3][3];  // c[d] = a_{d+1} x a_{d+2}
    cross(a[1], a[2], c[0]);
    cross(a[2], a[0], c[1]);
    cross(a[0], a[1], c[2]);
    const double vs = dot(a[0], c[0]);
    const double V = std::fabs(vs);
    if (!(V > 0) || !std::isfinite(V)) throw std::invalid_argument("degenerate cell");
    // fractional coordinates: s_d = (c_d . x) / (a_d . c_d)
    double ainv[9];
    for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 3; ++e) ainv[3 * d + e] = c[d][e] / vs;
    double h[3];
    for (int d = 0; d < 3; ++d) h[d] = V / std::sqrt(dot(c[d], c[d]));

    // parameters (cpp/src/ewald_nufft.cpp:40-56, 453-457)
    double target_nbr = 5000.0;
    if (const char* e = std::getenv("DMK_EWALD_TARGET_NBR")) target_nbr = std::atof(e);
    if (!(target_nbr > 0)) throw std::invalid_argument("DMK_EWALD_TARGET_NBR must be positive");
    const double alpha_bal = std::pow((double)n * M_PI * M_PI * M_PI / (V * V), 1.0 / 6.0);
    const double alpha_den = s * std::cbrt(4.0 * M_PI * ((double)n / V) / (3.0 * target_nbr));
    const double alpha = std::max(alpha_bal, alpha_den);
    const double rcut = s / alpha, kmax = 2.0 * s * alpha;

    // ---- real space: bins on fractional coordinates
    int m[3], R[3];
    for (int d = 0; d < 3; ++d) {
        m[d] = std::max(1, (int)std::floor(h[d] / rcut));
        m[d] = std::min(m[d], 1024);
        R[d] = (int)std::ceil(rcut * m[d] / h[d]);
    }
    const int64_t nbins = (int64_t)m[0] * m[1] * m[2];
    if (nbins > (1 << 26)) throw std::invalid_argument("too many real-space bins");
    if ((int64_t)(2 * R[0] + 1) * (2 * R[1] + 1) * (2 * R[2] + 1) > (1 << 20))
        throw std::invalid_argument("cell too thin for the real-space cutoff (more than 2^20 image bins per target)");
    std::vector<int> bin(n);
    std::vector<double4> wrapped(n);
    for (int i = 0; i < n; ++i) {
        const double* x = pos + 3 * (size_t)i;
        double fl[3];
        int id[3];
        for (int d = 0; d < 3; ++d) {
            const double sd = ainv[3 * d] * x[0] + ainv[3 * d + 1] * x[1] + ainv[3 * d + 2] * x[2];
            if (!std::isfinite(sd)) throw std::invalid_argument("non-finite position");
            fl[d] = std::floor(sd);
            id[d] = std::min(m[d] - 1, std::max(0, (int)((sd - fl[d]) * m[d])));
        }
        double w[3];
        for (int e = 0; e < 3; ++e) w[e] = x[e] - (fl[0] * a[0][e] + fl[1] * a[1][e] + fl[2] * a[2][e]);
        wrapped[i] = make_double4(w[0], w[1], w[2], q[i]);
        bin[i] = (id[0] * m[1] + id[1]) * m[2] + id[2];
    }
    std::vector<int> start(nbins + 1, 0);
    for (int i = 0; i < n; ++i) ++start[bin[i] + 1];
    std::partial_sum(start.begin(), start.end(), start.begin());
    std::vector<int> order(n), fill(start.begin(), start.end() - 1);
    for (int i = 0; i < n; ++i) order[fill[bin[i]]++] = i;
    std::vector<double4> sorted(n);
    for (int i = 0; i < n; ++i) sorted[i] = wrapped[order[i]];

    // ---- reciprocal grid (cpp/src/ewald_nufft.cpp:65-86): |m_d| <= ceil(kmax |a_d| / 2 pi)
    int mmax[3], ng[3];
    for (int d = 0; d < 3; ++d) {
        mmax[d] = (int)std::ceil(kmax * std::sqrt(dot(a[d], a[d])) / (2.0 * M_PI));
        ng[d] = smooth_size(std::max(2 * (2 * mmax[d] + 1), 2 * kEsW));
    }
    const int64_t ngrid = (int64_t)ng[0] * ng[1] * ng[2];
    const int n3h = ng[2] / 2 + 1;
    const int64_t nspec = (int64_t)ng[0] * ng[1] * n3h;
    if (ngrid > ((int64_t)1 << 31)) throw std::invalid_argument("reciprocal grid too large");
    // multiplier: w(K) (h0 h1 h2)^2 / (phihat0 phihat1 phihat2)^2 on the half spectrum
    const double beta = 2.30 * kEsW;
    std::vector<double> gx(200), gw(200);
    gauss_legendre(200, gx.data(), gw.data());
    std::vector<double> ph[3];
    for (int d = 0; d < 3; ++d) {
        const double hh = 2.0 * M_PI / ng[d], ah = 0.5 * kEsW * hh;
        ph[d].resize(ng[d]);
        for (int i = 0; i < ng[d]; ++i) {
            const int k = i <= ng[d] / 2 ? i : i - ng[d];
            double acc = 0.0;
            for (int j = 0; j < 200; ++j)
                acc += gw[j] * std::exp(beta * (std::sqrt(1.0 - gx[j] * gx[j]) - 1.0)) * std::cos(k * ah * gx[j]);
            ph[d][i] = ah * acc;
        }
    }
    double b[3][3];  // reciprocal vectors, b_d . a_e = 2 pi delta
    for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 3; ++e) b[d][e] = 2.0 * M_PI * c[d][e] / vs;
    const double H = std::pow(2.0 * M_PI, 3) / (double)ngrid;
    std::vector<double> mult(nspec, 0.0);
    for (int i0 = 0; i0 < ng[0]; ++i0)
        for (int i1 = 0; i1 < ng[1]; ++i1)
            for (int i2 = 0; i2 < n3h; ++i2) {
                const int k0 = i0 <= ng[0] / 2 ? i0 : i0 - ng[0];
                const int k1 = i1 <= ng[1] / 2 ? i1 : i1 - ng[1];
                const int k2 = i2;
                if (std::abs(k0) > mmax[0] || std::abs(k1) > mmax[1] || k2 > mmax[2]) continue;
                if (!k0 && !k1 && !k2) continue;
                double K[3];
                for (int e = 0; e < 3; ++e) K[e] = k0 * b[0][e] + k1 * b[1][e] + k2 * b[2][e];
                const double k2n = dot(K, K);
                if (k2n > kmax * kmax) continue;
                const double w = 4.0 * M_PI / V * std::exp(-k2n / (4.0 * alpha * alpha)) / k2n;
                const double P = ph[0][i0] * ph[1][i1] * ph[2][i2];
                mult[((size_t)i0 * ng[1] + i1) * n3h + i2] = w * H * H / (P * P);
            }

    // ---- device
    int dev_id = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev_id));
    cudaStream_t st = nullptr;
    PDMK_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            if (s) cudaStreamDestroy(s);
        }
    } sg{st};
    DevBuf<double4> d_pts(n);
    DevBuf<int> d_start(nbins + 1);
    DevBuf<double> d_real(n), d_far(n), d_grid(ngrid), d_mult(nspec);
    DevBuf<cd> d_spec(nspec);
    PDMK_CUDA_CHECK(cudaMemcpyAsync(d_pts.p, sorted.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, st));
    PDMK_CUDA_CHECK(cudaMemcpyAsync(d_start.p, start.data(), sizeof(int) * (nbins + 1), cudaMemcpyHostToDevice, st));
    PDMK_CUDA_CHECK(cudaMemcpyAsync(d_mult.p, mult.data(), sizeof(double) * nspec, cudaMemcpyHostToDevice, st));
    {
        RealArgs A{};
        A.pts = d_pts.p;
        A.bin_start = d_start.p;
        A.m0 = m[0]; A.m1 = m[1]; A.m2 = m[2];
        A.r0 = R[0]; A.r1 = R[1]; A.r2 = R[2];
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 3; ++e) A.a[3 * d + e] = a[d][e];
        A.alpha = alpha;
        A.rc2 = rcut * rcut;
        A.out = d_real.p;
        int maxc = 0;
        for (int64_t i = 0; i < nbins; ++i) maxc = std::max(maxc, start[i + 1] - start[i]);
        const int gy = std::max(1, std::min(64, (maxc + kRealThreads - 1) / kRealThreads));
        k_ewald_real<<<dim3((unsigned)nbins, gy), kRealThreads, 0, st>>>(A);
        PDMK_CUDA_CHECK(cudaGetLastError());
    }
    {
        NufftE E{};
        E.pts = d_pts.p;
        for (int i = 0; i < 9; ++i) E.ainv[i] = ainv[i];
        for (int d = 0; d < 3; ++d) E.n[d] = ng[d];
        E.beta = beta;
        E.grid = d_grid.p;
        E.out = d_far.p;
        E.npts = n;
        PDMK_CUDA_CHECK(cudaMemsetAsync(d_grid.p, 0, sizeof(double) * ngrid, st));
        const unsigned blocks = (unsigned)((n + 127) / 128);
        k_ewald_spread<<<blocks, 128, 0, st>>>(E);
        PDMK_CUDA_CHECK(cudaGetLastError());
        FftPlan fwd, inv;
        if (cufftPlan3d(&fwd.h, ng[0], ng[1], ng[2], CUFFT_D2Z) != CUFFT_SUCCESS ||
            cufftPlan3d(&inv.h, ng[0], ng[1], ng[2], CUFFT_Z2D) != CUFFT_SUCCESS)
            throw std::runtime_error("cuFFT error: Ewald plan creation failed");
        cufftSetStream(fwd.h, st);
        cufftSetStream(inv.h, st);
        if (cufftExecD2Z(fwd.h, d_grid.p, reinterpret_cast<cufftDoubleComplex*>(d_spec.p)) != CUFFT_SUCCESS)
            throw std::runtime_error("cuFFT error in the Ewald forward transform");
        k_ewald_scale<<<(unsigned)((nspec + 255) / 256), 256, 0, st>>>(d_spec.p, d_mult.p, nspec);
        if (cufftExecZ2D(inv.h, reinterpret_cast<cufftDoubleComplex*>(d_spec.p), d_grid.p) != CUFFT_SUCCESS)
            throw std::runtime_error("cuFFT error in the Ewald inverse transform");
        k_ewald_interp<<<blocks, 128, 0, st>>>(E);
        PDMK_CUDA_CHECK(cudaGetLastError());
    }
    std::vector<double> real(n), far(n);
    PDMK_CUDA_CHECK(cudaMemcpyAsync(real.data(), d_real.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    PDMK_CUDA_CHECK(cudaMemcpyAsync(far.data(), d_far.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    PDMK_CUDA_CHECK(cudaStreamSynchronize(st));
    double E = 0.0, Q = 0.0;
    const double self = 2.0 * alpha / std::sqrt(M_PI);
    for (int k = 0; k < n; ++k) {
        const int i = order[k];
        const double u = real[k] + far[k] - self * q[i];
        pot[i] = u;
        E += q[i] * u;
        Q += q[i];
    }
    if (energy) *energy = 0.5 * E - M_PI * Q * Q / (2.0 * V * alpha * alpha);
    if (info) {
        info->alpha = alpha;
        info->rcut = rcut;
        info->kmax = kmax;
        for (int d = 0; d < 3; ++d) {
            info->bins[d] = m[d];
            info->grid[d] = ng[d];
            info->modes[d] = 2 * mmax[d] + 1;
        }
    }
}

}  // namespace pdmkb
