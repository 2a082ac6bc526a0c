// Public C++ API: build-once / evaluate-many periodic Laplace (Coulomb) solver.
//
// Drop-in for the reference's PeriodicDMKTreeT<Real, DIM>
// (cpp/include/pdmk/periodic_dmk.hpp:17-60): same constructor arguments,
// evaluate / evaluate_timed semantics, n_points(), cube_size(); non-copyable,
// non-movable, not thread-safe.  Construction builds the tree on the host and
// uploads it to the current CUDA device; evaluate runs on that GPU.
//   Real = double : plain path, FP64 throughout.
//   Real = float  : mixed-precision path (FP32 near field and transforms where
//                   the error budget allows, FP64 far field and accumulation),
//                   float output as in the reference.
// With a Bloch vector (taken in the lattice-QR frame, as the reference takes
// it) the tree is quasi-periodic: evaluate_complex returns
// sum_j q_j sum_R e^{i bloch.R} G(x_i - x_j - R), computed in FP64 for both
// Real types, and evaluate / evaluate_timed / evaluate_multi throw
// std::logic_error.  Only DIM = 3 is provided (the reference's 2D path is not
// part of this build).
#pragma once
#include <array>
#include <complex>
#include <memory>
#include <optional>
#include <variant>
#include <vector>

#include "eval_timing.hpp"
#include "types.hpp"

namespace pdmk {

template <typename Real = double, int DIM = 3>
class PeriodicDMKTreeT {
    static_assert(DIM == 3, "only DIM = 3 is supported");

  public:
    using scalar_type = Real;

    PeriodicDMKTreeT(const MatND<DIM>& cell_matrix, const std::vector<VecND<DIM>>& positions, int n_digits = 6,
                     int n_per_leaf = 300, int nz = 4, std::optional<std::array<double, DIM>> bloch = std::nullopt);
    ~PeriodicDMKTreeT();
    PeriodicDMKTreeT(const PeriodicDMKTreeT&) = delete;
    PeriodicDMKTreeT& operator=(const PeriodicDMKTreeT&) = delete;
    PeriodicDMKTreeT(PeriodicDMKTreeT&&) = delete;
    PeriodicDMKTreeT& operator=(PeriodicDMKTreeT&&) = delete;

    /// Periodic Coulomb potentials sum'_{j,n} q_j / |x_i - x_j - R_n| at the
    /// stored positions (neutral gauge: the k = 0 mode is dropped).
    /// Throws std::invalid_argument if charges.size() != n_points().
    std::vector<Real> evaluate(const std::vector<double>& charges);
    /// Same, with a three-way device-time breakdown.
    std::vector<Real> evaluate_timed(const std::vector<double>& charges, EvalTiming& timing);
    /// k charge vectors on the same tree: charges is N x k column-major
    /// (charges[i + N*c]); returns N x k column-major potentials.
    std::vector<Real> evaluate_multi(const std::vector<double>& charges, int k);
    /// Quasi-periodic potentials (trees built with a Bloch vector; the
    /// reference's evaluate_complex, cpp/src/periodic_dmk.cpp:251-276).
    /// Throws std::logic_error without a Bloch vector, std::invalid_argument if
    /// charges.size() != n_points().
    std::vector<std::complex<Real>> evaluate_complex(const std::vector<double>& charges);

    int n_points() const { return n_src_; }
    double cube_size() const { return rc_; }

    struct Impl;
    Impl* impl() { return p_.get(); }

  private:
    std::unique_ptr<Impl> p_;
    int n_src_;
    double rc_;
    bool qp_ = false;
};

using PeriodicDMKTree = PeriodicDMKTreeT<double, 3>;

/// Float / double selection by digit count (drop-in for the reference's
/// AutoPeriodicDMKTree, cpp/include/pdmk/periodic_dmk.hpp:79-106, selection
/// rule cpp/src/periodic_dmk.cpp:326-336): the float tree (mixed-precision
/// path) for n_digits <= 6, the double tree (plain FP64 path) above.
using AnyPDMKTree = std::variant<std::unique_ptr<PeriodicDMKTreeT<float, 3>>,
                                 std::unique_ptr<PeriodicDMKTreeT<double, 3>>>;

class AutoPeriodicDMKTree {
  public:
    AutoPeriodicDMKTree(const Mat3& cell, const std::vector<Vec3>& positions, int n_digits, int n_per_leaf = 300,
                        int nz = 4);
    AutoPeriodicDMKTree(const AutoPeriodicDMKTree&) = delete;
    AutoPeriodicDMKTree& operator=(const AutoPeriodicDMKTree&) = delete;
    AutoPeriodicDMKTree(AutoPeriodicDMKTree&&) = default;
    AutoPeriodicDMKTree& operator=(AutoPeriodicDMKTree&&) = default;

    bool is_single_precision() const { return single_precision_; }
    /// float potentials from the float tree, double from the double tree
    std::variant<std::vector<float>, std::vector<double>> evaluate(const std::vector<double>& charges);

  private:
    AnyPDMKTree impl_;
    bool single_precision_ = false;
};

AutoPeriodicDMKTree make_periodic_dmk_tree(const Mat3& cell, const std::vector<Vec3>& positions, int n_digits,
                                           int n_per_leaf = 300, int nz = 4);

extern template class PeriodicDMKTreeT<double, 3>;
extern template class PeriodicDMKTreeT<float, 3>;

}  // namespace pdmk
