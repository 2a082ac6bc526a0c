// Prolate spheroidal wave function psi_0^c and Gauss-Legendre quadrature.
//
// Host-side precompute for the DMK split.  The reference builds psi_0 from the
// eigenvector of the prolate differential operator in the Legendre basis
// (cpp/src/dmk/prolate.cpp:348-449, prol0ini / prol0eva) and integrates it with
// Gauss-Legendre rules (cpp/src/dmk/legeexps.cpp:77-173, legerts).  This file
// computes the same function from the same mathematics: the symmetric
// tridiagonal operator matrix in the normalised even-Legendre basis is
// diagonalised by cyclic Jacobi rotations and the eigenvector of the smallest
// eigenvalue is normalised to unit L2 norm on [-1,1] with psi_0(0) > 0.
#pragma once
#include <vector>

namespace pdmkb {

// n-point Gauss-Legendre nodes (ascending) and weights on [-1, 1] (computed
// once per n and process; thread-safe).
void gauss_legendre(int n, double* x, double* w);

class Pswf0 {
  public:
    Pswf0() = default;
    explicit Pswf0(double c);
    // The function for c, built once per c and process (thread-safe; every
    // tree of a digit count shares it).
    static const Pswf0& get(double c);
    // psi_0^c(x) for |x| <= 1 (0 outside: the DMK tables never evaluate there).
    double operator()(double x) const;
    double c() const { return c_; }
    // Moments on [0,1] with a 200-point rule, as prolate_intvals
    // (cpp/src/dmk/prolate.cpp:483-511): c0 = int psi, c1 = int x psi,
    // c2 = int x^2 psi / c0, c4 = int x^4 psi.
    void moments(double& c0, double& c1, double& c2, double& c4) const;

  private:
    double c_ = 0;
    std::vector<double> leg_;  // Legendre coefficients of P_k, k = 0..K
    double mom_[4] = {0, 0, 0, 0};  // c0, c1, c2, c4 (computed by the constructor)
};

}  // namespace pdmkb
