// Quasi-periodic (Bloch) evaluate: u(x) = sum_j q_j sum_R e^{i bloch.R} G(x - x_j - R)
// (the reference's pbcdmk_adaptive with a Bloch vector, cpp/src/dmk/pbc.cpp:787-858).
//
// The tree part is linear in the charges with a real kernel, so it runs as two
// real right-hand sides of the FP64 multi-RHS path: the real and imaginary
// parts of the phased charges q_j e^{i bloch.R} of every source image.  The
// self term acts on the real part only (the original of a target has phase 1).
//
// The far field (cpp/src/dmk/pbc.cpp:250-357) weights the spectrum of the
// charges c_j = q_j e^{-i bloch.x_j} by w(K + bloch), which is not even in the
// mode k, so the spectrum is not Hermitian.  With c = a + i b split into two
// real grids whose transforms A, B are Hermitian, the weighted spectrum
// G = w (A + i B) has real-grid parts
//   P = s A + i d B,  Q = s B - i d A,  s = (w(k) + w(-k))/2, d = (w(k) - w(-k))/2
// (P(k) = (G(k) + conj G(-k))/2, Q(k) = (G(k) - conj G(-k))/(2i)), which the
// two real inverse transforms take back to the real and imaginary parts of the
// far-field sum; the potential is e^{i bloch.x} (P + i Q) at the target.
#include <cuda_runtime.h>

#include "qp.cuh"

namespace pdmkb {
namespace dev {

namespace {

__global__ void k_qp_src_rows(double* __restrict__ src_q, const int* __restrict__ idx,
                              const double2* __restrict__ ph, const double* __restrict__ q, int64_t n_all) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_all) return;
    const double c = q[idx[j]];
    const double2 e = ph[j];
    reinterpret_cast<double2*>(src_q)[j] = make_double2(c * e.x, c * e.y);
}

__global__ void k_qp_far_q(double* __restrict__ far_q, const int* __restrict__ perm, const double2* __restrict__ ph,
                           const double* __restrict__ q, int64_t n) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double c = q[perm[t]];
    const double2 e = ph[t];
    far_q[t] = c * e.x;
    far_q[n + t] = -c * e.y;
}

__global__ void k_qp_combine(cd* __restrict__ spec, const double* __restrict__ qs, const double* __restrict__ qd,
                             int64_t n_spec) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_spec) return;
    const cd a = spec[i], b = spec[n_spec + i];
    const double sv = qs[i], dv = qd[i];
    spec[i] = {sv * a.x - dv * b.y, sv * a.y + dv * b.x};
    spec[n_spec + i] = {sv * b.x + dv * a.y, sv * b.y - dv * a.x};
}

__global__ void k_qp_finalize(const double* __restrict__ pot, const double* __restrict__ far,
                              const double4* __restrict__ trg, const int* __restrict__ perm,
                              const double* __restrict__ q, const double2* __restrict__ ph, double* __restrict__ out,
                              int64_t n) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int u = perm[t];
    const double2 e = ph[t];
    const double fr = far[t], fi = far[n + t];
    const double re = pot[t] - trg[t].w * q[u] + (e.x * fr - e.y * fi);
    const double im = pot[n + t] + (e.y * fr + e.x * fi);
    out[2 * (int64_t)u] = re;  // the caller's buffer may be only 8-byte aligned
    out[2 * (int64_t)u + 1] = im;
}

inline unsigned blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

}  // namespace

void launch_qp_charges(double* src_q, const int* idx, const double2* src_phase, int64_t n_all, double* far_q,
                       const int* perm, const double2* trg_phase, int64_t n, const double* q, cudaStream_t s) {
    if (n_all > 0) k_qp_src_rows<<<blocks(n_all), 256, 0, s>>>(src_q, idx, src_phase, q, n_all);
    if (n > 0) k_qp_far_q<<<blocks(n), 256, 0, s>>>(far_q, perm, trg_phase, q, n);
}

void launch_qp_combine(cd* spec, const double* qs, const double* qd, int64_t n_spec, cudaStream_t s) {
    if (n_spec > 0) k_qp_combine<<<blocks(n_spec), 256, 0, s>>>(spec, qs, qd, n_spec);
}

void launch_qp_finalize(const double* pot, const double* far, const double4* trg, const int* perm, const double* q,
                        const double2* trg_phase, double* out, int64_t n, cudaStream_t s) {
    if (n > 0) k_qp_finalize<<<blocks(n), 256, 0, s>>>(pot, far, trg, perm, q, trg_phase, out, n);
}

}  // namespace dev
}  // namespace pdmkb
