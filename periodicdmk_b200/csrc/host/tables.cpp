// Precomputed tables of the evaluate path (host, once per tree).
//
//   Chebyshev nodes / parent<->child maps   cpp/include/dmk/chebychev.hpp:38-302
//   poly2pw / pw2poly                        cpp/src/dmk/planewave.cpp:118-146
//   translation (shift) matrices             cpp/src/dmk/planewave.cpp:148-223
//   difference-kernel FT, Laplace 3D         cpp/src/dmk/fourier_data.cpp:415-463, 863-887
//   tensor-product FT layout                 cpp/src/dmk/util.cpp:126-141
//   kernel FT fused into shifts              cpp/src/dmk/pbc_tree.cpp:1013-1103
//   self-interaction constant                cpp/include/dmk/tree.hpp:348-387
//   periodic far-field weights               cpp/src/dmk/pbc.cpp:386-438
#include <cmath>
#include <vector>

#include "plan.hpp"
#include "pswf.hpp"

namespace pdmkb {

namespace {

// Chebyshev nodes on [-1,1] in ascending order.
std::vector<double> cheb_nodes(int p) {
    std::vector<double> x(p);
    for (int i = 0; i < p; ++i) x[i] = std::cos(M_PI * ((p - i - 1) + 0.5) / p);
    return x;
}

// T_a(x) for a = 0..p-1.
void cheb_T(int p, double x, double* t) {
    t[0] = 1.0;
    if (p > 1) t[1] = x;
    for (int a = 2; a < p; ++a) t[a] = 2.0 * x * t[a - 1] - t[a - 2];
}

// Inverse of the Vandermonde V(i,a) = T_a(x_i) at the Chebyshev nodes, by
// discrete orthogonality: Vinv(a,i) = (2 - delta_a0)/p * T_a(x_i).
// Returned column-major p x p: vinv[a + p*i].
std::vector<double> cheb_vinv(int p) {
    const auto x = cheb_nodes(p);
    std::vector<double> vinv((size_t)p * p), t(p);
    for (int i = 0; i < p; ++i) {
        cheb_T(p, x[i], t.data());
        for (int a = 0; a < p; ++a) vinv[a + (size_t)p * i] = (a == 0 ? 1.0 : 2.0) / p * t[a];
    }
    return vinv;
}

}  // namespace

void build_tables(Plan& P) {
    const int p = P.p, n = P.n_pw, n2 = P.n_pw2, M = P.n_modes;
    const double beta = P.dp.beta;
    const Pswf0& pf = Pswf0::get(beta);
    double c0, c1, c2, c4;
    pf.moments(c0, c1, c2, c4);
    const double psi0 = pf(0.0);
    P.psi0_at_zero = psi0;
    P.c0 = c0;

    // ---- self-interaction constants: W_b(0) = psi0 / (c0 * b), with the
    // level-0 entry using b = rc/2 as the reference does.
    P.w0.assign(P.nlevels + 1, 0.0);
    for (int d = 0; d <= P.nlevels; ++d) {
        const double bs = d == 0 ? 0.5 * P.boxsize[0] : P.boxsize[d];
        P.w0[d] = psi0 / (c0 * bs);
    }

    // ---- parent -> child coefficient maps: P_pm = Vinv * V(x/2 -+ 1/2)
    const auto vinv = cheb_vinv(p);
    const auto xs = cheb_nodes(p);
    std::vector<double> pm[2];
    for (int side = 0; side < 2; ++side) {
        pm[side].assign((size_t)p * p, 0.0);
        std::vector<double> t(p);
        // V_side(i, b) = T_b(0.5 x_i + (side ? 0.5 : -0.5))
        std::vector<double> vs((size_t)p * p);
        for (int i = 0; i < p; ++i) {
            cheb_T(p, 0.5 * xs[i] + (side ? 0.5 : -0.5), t.data());
            for (int b = 0; b < p; ++b) vs[i + (size_t)p * b] = t[b];
        }
        for (int a = 0; a < p; ++a)
            for (int b = 0; b < p; ++b) {
                double s = 0;
                for (int i = 0; i < p; ++i) s += vinv[a + (size_t)p * i] * vs[i + (size_t)p * b];
                pm[side][a + (size_t)p * b] = s;
            }
    }
    // Child c (bit d set = upper half along dim d) uses P_{bit d} along dim d.
    P.p2c.assign((size_t)8 * 3 * p * p, 0.0);
    for (int c = 0; c < 8; ++c)
        for (int d = 0; d < 3; ++d) {
            const auto& m = pm[(c >> d) & 1];
            std::copy(m.begin(), m.end(), P.p2c.begin() + ((size_t)c * 3 + d) * p * p);
        }

    // ---- difference kernel FT at level 0 (radial, indexed by |k_int|^2)
    const int nf = (n - 1) / 2;
    const int n_fourier = 3 * (n / 2) * (n / 2) + 1;
    std::vector<double> gx(100), gw(100);
    gauss_legendre(100, gx.data(), gw.data());
    std::vector<double> kft(n_fourier);
    {
        const double bsmall = 0.5 * P.boxsize[0], bbig = P.boxsize[0];
        const double hpw = 2.0 * beta / nf / P.boxsize[0];
        const double ws = hpw * hpw * hpw * 0.5 / (M_PI * M_PI);
        std::vector<double> x1(100), x2(100), fv(100);
        for (int i = 0; i < 100; ++i) {
            const double t = 0.5 * (gx[i] + 1.0);
            x1[i] = t * bsmall;
            x2[i] = t * bbig;
            fv[i] = 0.5 * pf(t) * gw[i] / c0;
        }
        for (int i = 0; i < n_fourier; ++i) {
            if (i == 0) {
                kft[0] = 0.5 * ws * c2 * (bbig * bbig - bsmall * bsmall);
                continue;
            }
            const double rk = std::sqrt((double)i) * hpw;
            double s = 0;
            for (int j = 0; j < 100; ++j) s += (std::cos(rk * x1[j]) - std::cos(rk * x2[j])) * fv[j];
            kft[i] = s * ws / (rk * rk);
        }
    }

    // ---- per-level plane-wave tables
    P.lev.assign(P.nlevels, {});
    const int shift = n / 2;
    for (int l = 0; l < P.nlevels; ++l) {
        auto& T = P.lev[l];
        const double bs = P.boxsize[l];
        T.hpw = 2.0 * beta / nf / bs;
        if (l > 0)
            for (double& v : kft) v *= 2.0;  // D_l(k) = 2^l D_0 on the integer mode grid
        // pw2poly(j,a) = Chebyshev coefficient a of exp(i t_j (bs/2) x) on [-1,1]
        T.pw2poly.assign((size_t)n * p, cplx(0));
        T.poly2pw.assign((size_t)n * p, cplx(0));
        for (int j = 0; j < n; ++j)
            for (int a = 0; a < p; ++a) {
                cplx s(0);
                for (int i = 0; i < p; ++i) {
                    const double ph = (j - shift) * xs[i] * 0.5 * bs * T.hpw;
                    s += vinv[a + (size_t)p * i] * cplx(std::cos(ph), std::sin(ph));
                }
                T.pw2poly[j + (size_t)n * a] = s;
                T.poly2pw[j + (size_t)n * a] = std::conj(s);
            }
        // radial FT in the (k1 fastest, k2, k3 half-space) mode layout
        T.radialft.resize(M);
        {
            int ind = 0;
            for (int j3 = -n / 2; j3 <= 0; ++j3)
                for (int j2 = -n / 2; j2 <= (n - 1) / 2; ++j2)
                    for (int j1 = -n / 2; j1 <= (n - 1) / 2; ++j1) T.radialft[ind++] = kft[j1 * j1 + j2 * j2 + j3 * j3];
        }
        // 27 translation stencils: stencil s = kx + 3 ky + 9 kz, offset
        // (k - 1) * bs between box centres; factor exp(i t (k-1) bs) per axis,
        // multiplied by the radial kernel FT.
        T.shift.assign((size_t)27 * 2 * M, 0.0);
        std::vector<cplx> ww((size_t)n * 3);
        for (int j = 0; j < n; ++j) {
            const double ts = (j - shift) * T.hpw;
            const cplx base(std::cos(ts * bs), std::sin(ts * bs));
            ww[j + n * 0] = std::conj(base);
            ww[j + n * 1] = 1.0;
            ww[j + n * 2] = base;
        }
        for (int s = 0; s < 27; ++s) {
            const int kx = s % 3, ky = (s / 3) % 3, kz = s / 9;
            double* re = &T.shift[(size_t)s * 2 * M];
            double* im = re + M;
            int m = 0;
            for (int j0 = 0; j0 < n2; ++j0)
                for (int j1 = 0; j1 < n; ++j1)
                    for (int j2 = 0; j2 < n; ++j2, ++m) {
                        const cplx v = ww[j0 + n * kz] * ww[j1 + n * ky] * ww[j2 + n * kx];
                        re[m] = v.real() * T.radialft[m];
                        im[m] = v.imag() * T.radialft[m];
                    }
        }
    }

    P.resid = residual_coeffs(P.dp.n_digits_tree);

    // ---- periodic far field: W_rc on the reciprocal lattice
    {
        const double twopi = 2.0 * M_PI;
        const double* u = P.umat;
        // quasi-periodic: the modes reach |2 pi L^-T m + bloch| <= beta / rc
        // (cpp/src/dmk/pbc.cpp:258-265)
        const double bn = P.qp ? std::sqrt(P.bloch[0] * P.bloch[0] + P.bloch[1] * P.bloch[1] + P.bloch[2] * P.bloch[2])
                               : 0.0;
        const double dkmax = beta / P.rc + bn;
        const double an1 = u[0];
        const double an2 = std::sqrt(u[3] * u[3] + u[4] * u[4]);
        const double an3 = std::sqrt(u[6] * u[6] + u[7] * u[7] + u[8] * u[8]);
        P.ms = std::max(2, 2 * (int)std::ceil(dkmax * an1 / twopi));
        P.mt = std::max(2, 2 * (int)std::ceil(dkmax * an2 / twopi));
        P.mu = std::max(2, 2 * (int)std::ceil(dkmax * an3 / twopi));
        const double a11 = 1.0 / u[0], a21 = -u[3] / (u[0] * u[4]), a22 = 1.0 / u[4];
        const double a31 = (u[3] * u[7] - u[6] * u[4]) / (u[0] * u[4] * u[8]);
        const double a32 = -u[7] / (u[4] * u[8]), a33 = 1.0 / u[8];
        const double dfac = 4.0 * M_PI / (psi0 * P.volume);
        P.ff_weights.assign((size_t)P.ms * P.mt * P.mu, 0.0);
        size_t idx = 0;
        for (int k = -P.mu / 2; k <= (P.mu - 1) / 2; ++k)
            for (int j = -P.mt / 2; j <= (P.mt - 1) / 2; ++j)
                for (int i = -P.ms / 2; i <= (P.ms - 1) / 2; ++i, ++idx) {
                    // shifted wavenumbers 2 pi L^-T m + bloch (bloch = 0 when periodic)
                    const double d1 = twopi * (a11 * i) + P.bloch[0];
                    const double d2 = twopi * (a21 * i + a22 * j) + P.bloch[1];
                    const double d3 = twopi * (a31 * i + a32 * j + a33 * k) + P.bloch[2];
                    const double k2 = d1 * d1 + d2 * d2 + d3 * d3;
                    if (k2 < 1e-30) continue;
                    const double xval = std::sqrt(k2) * P.rc / beta;
                    const double f = xval <= 1.0 ? pf(xval) : 0.0;
                    P.ff_weights[idx] = dfac * f / k2;
                }
    }
}

}  // namespace pdmkb
