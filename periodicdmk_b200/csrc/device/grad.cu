// Gradient of the potential at the targets, plain FP64 path (the reference's
// target gradients: eval_targets with derivative tables, cpp/src/dmk/proxy.cpp:307-448,
// and the has_grad branches of the residual kernel,
// cpp/include/dmk/vector_kernels.hpp:391-417; pgh_trg = DMK_POTENTIAL_GRAD):
//   * near field: R_b(r) = P(x)/r, x = (r - b/2) 2/b, so dR/dr = P'(x) (2/b)/r - P(x)/r^2,
//     the gradient at the target is dR/dr (t - s)/r; P and P' come from one Horner pass;
//   * leaf evaluation: u = sum C_ijk T_i(x') T_j(y') T_k(z'), x' = (x - c) s, so the
//     x-derivative is s sum C_ijk T_i'(x') T_j T_k with T_n' from the recurrence
//     T_{n+1}' = 2 T_n + 2 x T_n' - T_{n-1}';
//   * far field: spectral differentiation of the windowed far field: the
//     spectrum after the multiplier times i K_d, K = 2 pi L^-T k in the tree's
//     frame, one inverse transform and one interpolation per component;
//   * the self term (w0 q) has no gradient.
// Gradients are accumulated per sorted target in the tree's (rotated) frame,
// component-major (g[d * n + t]); the final gather rotates them back to the
// caller's frame (x = Q r, so grad_x = Q grad_r) and scatters to user order.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>

#include "common.cuh"
#include "grad.cuh"

namespace pdmkb {
namespace dev {

namespace {

template <int NC>
__global__ void __launch_bounds__(128) k_near_pg(NearArgs a, double* __restrict__ g, int64_t n) {
    constexpr int CH = 64;
    __shared__ double4 ss[CH];
    const int e = blockIdx.x;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    double c[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i) c[i] = a.coef[i];
    for (int base = 0; base < nt; base += 128) {
        const int t = base + threadIdx.x;
        const double4 tp = t < nt ? a.trg[t0 + t] : make_double4(1e300, 1e300, 1e300, 0.0);
        double acc = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
        for (int pr = a.pair_start[e]; pr < a.pair_start[e + 1]; ++pr) {
            const int s0 = a.pair_src_start[pr], ns = a.pair_src_count[pr];
            const double b = a.pair_bsize[pr];
            const double d2max = b * b, rsc = 2.0 / b, cen = -0.5 * b;
            for (int sb = 0; sb < ns; sb += CH) {
                __syncthreads();
                if ((int)threadIdx.x < CH && sb + (int)threadIdx.x < ns) ss[threadIdx.x] = a.src[s0 + sb + threadIdx.x];
                __syncthreads();
                const int m = min(CH, ns - sb);
                for (int j = 0; j < m; ++j) {
                    const double4 y = ss[j];
                    const double dx = tp.x - y.x, dy = tp.y - y.y, dz = tp.z - y.z;
                    const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
                    if (r2 > 1e-30 && r2 < d2max) {
                        const double rinv = rsqrt_nr(r2);  // as the potential-only near field
                        const double x = fma(r2, rinv, cen) * rsc;
                        double pv = c[NC - 1], dv = 0.0;
#pragma unroll
                        for (int i = NC - 2; i >= 0; --i) {
                            dv = fma(dv, x, pv);
                            pv = fma(pv, x, c[i]);
                        }
                        acc = fma(y.w * pv, rinv, acc);
                        // dR/dr / r = (P' rsc - P rinv) rinv^2
                        const double f = y.w * (dv * rsc - pv * rinv) * rinv * rinv;
                        gx = fma(f, dx, gx);
                        gy = fma(f, dy, gy);
                        gz = fma(f, dz, gz);
                    }
                }
            }
        }
        if (t < nt) {
            a.pot[t0 + t] += acc;
            g[t0 + t] += gx;
            g[n + t0 + t] += gy;
            g[2 * n + t0 + t] += gz;
        }
    }
}

// leaf evaluation gradient; per-thread Chebyshev tables of x in shared memory
// ([P][128], thread-fastest), the coefficient slab of one k in shared memory
template <int P>
__global__ void __launch_bounds__(128) k_eval_grad(EvalArgs a, double* __restrict__ g, int64_t n) {
    extern __shared__ double sme[];
    double* slab = sme;                 // P * P
    double* T = slab + P * P;           // [P][128]
    double* D = T + P * 128;            // [P][128]
    const int e = blockIdx.x, tid = threadIdx.x;
    const int t0 = a.trg_start[e], nt = a.trg_count[e];
    const double4 cs = a.center_scale[e];
    const double* C = a.proxy_down + (int64_t)a.slot[e] * (P * P * P);
    for (int base = 0; base < nt; base += 128) {
        const int t = base + tid;
        const bool act = t < nt;
        double x = 0.0, y = 0.0, z = 0.0;
        if (act) {
            const double4 pt = a.trg[t0 + t];
            x = (pt.x - cs.x) * cs.w;
            y = (pt.y - cs.y) * cs.w;
            z = (pt.z - cs.z) * cs.w;
        }
        {
            double t0v = 1.0, t1v = x, d0 = 0.0, d1 = 1.0;
            T[tid] = t0v;
            D[tid] = d0;
            if (P > 1) {
                T[128 + tid] = t1v;
                D[128 + tid] = d1;
            }
            for (int i = 2; i < P; ++i) {
                const double t2 = 2.0 * x * t1v - t0v, dd2 = 2.0 * t1v + 2.0 * x * d1 - d0;
                T[i * 128 + tid] = t2;
                D[i * 128 + tid] = dd2;
                t0v = t1v;
                t1v = t2;
                d0 = d1;
                d1 = dd2;
            }
        }
        double gx = 0.0, gy = 0.0, gz = 0.0;
        double za = 1.0, zb = z, dza = 0.0, dzb = 1.0;
        for (int k = 0; k < P; ++k) {
            __syncthreads();
            for (int idx = tid; idx < P * P; idx += 128) slab[idx] = C[(int64_t)k * P * P + idx];
            __syncthreads();
            double ya = 1.0, yb = y, dya = 0.0, dyb = 1.0;
            double sk = 0.0, sdx = 0.0, sdy = 0.0;
            for (int j = 0; j < P; ++j) {
                double r = 0.0, rd = 0.0;
                for (int i = 0; i < P; ++i) {
                    const double cij = slab[i + P * j];
                    r = fma(cij, T[i * 128 + tid], r);
                    rd = fma(cij, D[i * 128 + tid], rd);
                }
                sk = fma(ya, r, sk);
                sdx = fma(ya, rd, sdx);
                sdy = fma(dya, r, sdy);
                const double yn = 2.0 * y * yb - ya, dyn = 2.0 * yb + 2.0 * y * dyb - dya;
                ya = yb;
                yb = yn;
                dya = dyb;
                dyb = dyn;
            }
            gx = fma(za, sdx, gx);
            gy = fma(za, sdy, gy);
            gz = fma(dza, sk, gz);
            const double zn = 2.0 * z * zb - za, dzn = 2.0 * zb + 2.0 * z * dzb - dza;
            za = zb;
            zb = zn;
            dza = dzb;
            dzb = dzn;
        }
        if (act) {
            g[t0 + t] += cs.w * gx;
            g[n + t0 + t] += cs.w * gy;
            g[2 * n + t0 + t] += cs.w * gz;
        }
    }
}

// out = i K_d in over the half spectrum [n1][n2][n3/2 + 1]; v = upper-triangular
// inverse of the cell's R factor (column-major), K = 2 pi (k0 v0, k0 v3 + k1 v4,
// k0 v6 + k1 v7 + k2 v8) for integer modes (k0, k1, k2)
__global__ void k_grad_multiply(const cd* __restrict__ in, cd* __restrict__ out, int n1, int n2, int n3, int d,
                                GradFrame f) {
    const int n3h = n3 / 2 + 1;
    const int64_t tot = (int64_t)n1 * n2 * n3h;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tot) return;
    const int i3 = (int)(i % n3h);
    const int i2 = (int)((i / n3h) % n2);
    const int i1 = (int)(i / ((int64_t)n3h * n2));
    const double k0 = i1 <= n1 / 2 ? i1 : i1 - n1;
    const double k1 = i2 <= n2 / 2 ? i2 : i2 - n2;
    const double k2 = i3;
    const double* v = f.umatinv;
    const double twopi = 6.283185307179586476925286766559;
    const double K = d == 0 ? twopi * (k0 * v[0]) : d == 1 ? twopi * (k0 * v[3] + k1 * v[4])
                                                         : twopi * (k0 * v[6] + k1 * v[7] + k2 * v[8]);
    const cd a = in[i];
    out[i] = cd{-K * a.y, K * a.x};
}

__global__ void k_finalize_grad(const double* __restrict__ g, const double* __restrict__ far_g,
                                const int* __restrict__ perm, double* __restrict__ out, int64_t n, GradFrame f) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double r[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) r[d] = g[d * n + t] + far_g[d * n + t];
    const int u = perm[t];
#pragma unroll
    for (int e = 0; e < 3; ++e)
        out[3 * (int64_t)u + e] = f.qmat[e] * r[0] + f.qmat[e + 3] * r[1] + f.qmat[e + 6] * r[2];
}

}  // namespace

void launch_near_pg(const NearArgs& a, double* grad, int64_t n, cudaStream_t s) {
    if (a.n_leaves <= 0) return;
    switch (a.nc) {
#define PDMK_NPG(NC) \
    case NC: k_near_pg<NC><<<a.n_leaves, 128, 0, s>>>(a, grad, n); break;
        PDMK_NPG(5) PDMK_NPG(6) PDMK_NPG(9) PDMK_NPG(11) PDMK_NPG(12) PDMK_NPG(15) PDMK_NPG(17) PDMK_NPG(18)
        PDMK_NPG(22) PDMK_NPG(23) PDMK_NPG(25)
#undef PDMK_NPG
        default: throw std::runtime_error("unsupported residual polynomial length");
    }
}

template <int P>
static void launch_eg(const EvalArgs& a, double* grad, int64_t n, cudaStream_t s) {
    const size_t smem = sizeof(double) * ((size_t)P * P + 2 * (size_t)P * 128);
    static bool configured[64] = {};
    int dev = 0;
    PDMK_CUDA_CHECK(cudaGetDevice(&dev));
    if (!configured[dev & 63]) {
        PDMK_CUDA_CHECK(cudaFuncSetAttribute(k_eval_grad<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured[dev & 63] = true;
    }
    k_eval_grad<P><<<a.n_leaves, 128, smem, s>>>(a, grad, n);
}

void launch_eval_grad(const EvalArgs& a, int p, double* grad, int64_t n, cudaStream_t s) {
    if (a.n_leaves <= 0) return;
    switch (p) {
        case 9: launch_eg<9>(a, grad, n, s); break;
        case 18: launch_eg<18>(a, grad, n, s); break;
        case 28: launch_eg<28>(a, grad, n, s); break;
        case 38: launch_eg<38>(a, grad, n, s); break;
        default: throw std::runtime_error("unsupported expansion order");
    }
}

void launch_grad_multiply(const cd* spec, cd* out, int n1, int n2, int n3, int d, const GradFrame& f, cudaStream_t s) {
    const int64_t tot = (int64_t)n1 * n2 * (n3 / 2 + 1);
    if (tot <= 0) return;
    k_grad_multiply<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(spec, out, n1, n2, n3, d, f);
}

void launch_finalize_grad(const double* g, const double* far_g, const int* perm, double* out, int64_t n,
                          const GradFrame& f, cudaStream_t s) {
    if (n <= 0) return;
    k_finalize_grad<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, far_g, perm, out, n, f);
}

}  // namespace dev
}  // namespace pdmkb
