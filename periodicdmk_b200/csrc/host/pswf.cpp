#include "pswf.hpp"

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>

namespace pdmkb {

// Legendre P_n(x) and P_n'(x) by the three-term recurrence.
static void legendre_pd(int n, double x, double& p, double& dp) {
    double p0 = 1.0, p1 = x;
    if (n == 0) { p = 1.0; dp = 0.0; return; }
    for (int k = 2; k <= n; ++k) {
        double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = pk;
    }
    p = p1;
    dp = n * (x * p1 - p0) / (x * x - 1.0);
}

namespace {

void gauss_legendre_compute(int n, double* x, double* w) {
    // Newton iteration from the Tricomi initial guess; symmetric fill.
    const int m = (n + 1) / 2;
    for (int i = 0; i < m; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double p = 0, dp = 1;
        for (int it = 0; it < 100; ++it) {
            legendre_pd(n, z, p, dp);
            double dz = p / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-17) break;
        }
        legendre_pd(n, z, p, dp);
        const double wt = 2.0 / ((1.0 - z * z) * dp * dp);
        x[n - 1 - i] = z;
        x[i] = -z;
        w[n - 1 - i] = wt;
        w[i] = wt;
    }
    if (n % 2 == 1) x[m - 1] = 0.0;
}

}  // namespace

void gauss_legendre(int n, double* x, double* w) {
    static std::mutex mu;
    static std::map<int, std::pair<std::vector<double>, std::vector<double>>> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto& e = cache[n];
    if (e.first.empty() && n > 0) {
        e.first.resize(n);
        e.second.resize(n);
        gauss_legendre_compute(n, e.first.data(), e.second.data());
    }
    std::copy(e.first.begin(), e.first.end(), x);
    std::copy(e.second.begin(), e.second.end(), w);
}

// Cyclic Jacobi eigen-decomposition of a dense symmetric matrix (row-major).
// On return a holds the eigenvalues on its diagonal and v the eigenvectors
// as columns.
static void jacobi_eigen(int n, std::vector<double>& a, std::vector<double>& v) {
    v.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0, diag = 0;
        for (int i = 0; i < n; ++i) {
            diag += a[(size_t)i * n + i] * a[(size_t)i * n + i];
            for (int j = i + 1; j < n; ++j) off += a[(size_t)i * n + j] * a[(size_t)i * n + j];
        }
        if (off <= 1e-40 * diag) break;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                const double apq = a[(size_t)p * n + q];
                if (apq == 0.0) continue;
                const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
                    a[(size_t)k * n + p] = c * akp - s * akq;
                    a[(size_t)k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
                    a[(size_t)p * n + k] = c * apk - s * aqk;
                    a[(size_t)q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
                    v[(size_t)k * n + p] = c * vkp - s * vkq;
                    v[(size_t)k * n + q] = s * vkp + c * vkq;
                }
            }
        }
    }
}

Pswf0::Pswf0(double c) : c_(c) {
    // psi_0 is even: expand in normalised even Legendre functions
    // Pbar_k = sqrt(k + 1/2) P_k, k = 2r.  The prolate operator
    // L = -(d/dx)(1-x^2)(d/dx) + c^2 x^2 is symmetric tridiagonal there:
    //   diag:  k(k+1) + c^2 (2k^2+2k-1)/((2k-1)(2k+3))
    //   off:   c^2 (k+1)(k+2)/((2k+3) sqrt((2k+1)(2k+5)))
    const int m = std::max(40, (int)std::ceil(c) + 40);
    std::vector<double> a((size_t)m * m, 0.0), v;
    const double c2 = c * c;
    for (int r = 0; r < m; ++r) {
        const double k = 2.0 * r;
        a[(size_t)r * m + r] = k * (k + 1) + c2 * (2 * k * k + 2 * k - 1) / ((2 * k - 1) * (2 * k + 3));
        if (r + 1 < m) {
            const double off = c2 * (k + 1) * (k + 2) / ((2 * k + 3) * std::sqrt((2 * k + 1) * (2 * k + 5)));
            a[(size_t)r * m + r + 1] = off;
            a[(size_t)(r + 1) * m + r] = off;
        }
    }
    jacobi_eigen(m, a, v);
    int imin = 0;
    for (int r = 1; r < m; ++r)
        if (a[(size_t)r * m + r] < a[(size_t)imin * m + imin]) imin = r;
    std::vector<double> ev(m);
    double nrm = 0;
    for (int r = 0; r < m; ++r) {
        ev[r] = v[(size_t)r * m + imin];
        nrm += ev[r] * ev[r];
    }
    nrm = std::sqrt(nrm);
    leg_.assign(2 * m, 0.0);
    for (int r = 0; r < m; ++r) leg_[2 * r] = ev[r] / nrm * std::sqrt(2.0 * r + 0.5);
    // Fix the sign so that psi_0(0) > 0.
    if ((*this)(0.0) < 0)
        for (double& x : leg_) x = -x;
    // Drop the negligible tail.
    int last = (int)leg_.size() - 1;
    while (last > 0 && std::fabs(leg_[last]) < 1e-18 * std::fabs(leg_[0])) --last;
    leg_.resize(last + 1);
    // moments on [0,1] with a 200-point rule, as prolate_intvals
    // (cpp/src/dmk/prolate.cpp:483-511)
    const int nq = 200;
    std::vector<double> x(nq), w(nq);
    gauss_legendre(nq, x.data(), w.data());
    double s0 = 0, s1 = 0, s2 = 0, s4 = 0;
    for (int i = 0; i < nq; ++i) {
        const double t = 0.5 * (x[i] + 1.0), wt = 0.5 * w[i];
        const double f = (*this)(t);
        s0 += wt * f;
        s1 += wt * f * t;
        s2 += wt * f * t * t;
        s4 += wt * f * t * t * t * t;
    }
    mom_[0] = s0;
    mom_[1] = s1;
    mom_[2] = s2 / s0;
    mom_[3] = s4;
}

const Pswf0& Pswf0::get(double c) {
    static std::mutex mu;
    static std::map<double, std::unique_ptr<Pswf0>> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto& p = cache[c];
    if (!p) p = std::make_unique<Pswf0>(c);
    return *p;
}

double Pswf0::operator()(double x) const {
    if (std::fabs(x) > 1.0) return 0.0;
    double p0 = 1.0, p1 = x;
    double s = leg_[0];
    if (leg_.size() > 1) s += leg_[1] * x;
    for (size_t k = 2; k < leg_.size(); ++k) {
        const double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / (double)k;
        s += leg_[k] * pk;
        p0 = p1;
        p1 = pk;
    }
    return s;
}

void Pswf0::moments(double& c0, double& c1, double& c2, double& c4) const {
    c0 = mom_[0];
    c1 = mom_[1];
    c2 = mom_[2];
    c4 = mom_[3];
}

}  // namespace pdmkb
