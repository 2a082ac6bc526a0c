// PeriodicDMKTreeT<Real, 3>: host construction + GPU evaluate.
//
// Construction follows the reference's Impl constructor
// (cpp/src/periodic_dmk.cpp:41-139): parameters from n_digits, lattice QR,
// rc = min diag(umat) / nz, rotation of the positions into the umat frame,
// lattice images, tree.  All of that is the host plan builder; the resulting
// plan is uploaded once.  evaluate (cpp/src/periodic_dmk.cpp:141-186) runs
// entirely on the GPU.
#include "pdmk/periodic_dmk.hpp"

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "../device/device_tree.hpp"
#include "../device/tree_build.hpp"
#include "../host/plan.hpp"
#include "impl.hpp"

namespace pdmk {

template <typename Real, int DIM>
PeriodicDMKTreeT<Real, DIM>::PeriodicDMKTreeT(const MatND<DIM>& cell, const std::vector<VecND<DIM>>& positions,
                                              int n_digits, int n_per_leaf, int nz,
                                              std::optional<std::array<double, DIM>> bloch) {
    p_ = std::make_unique<Impl>();
    double c[9];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) c[j * 3 + i] = cell[j][i];
    std::vector<double> pos(3 * positions.size());
    for (size_t i = 0; i < positions.size(); ++i)
        for (int d = 0; d < 3; ++d) pos[3 * i + d] = positions[i][d];
    double b[3] = {0.0, 0.0, 0.0};
    if (bloch.has_value())
        for (int d = 0; d < 3; ++d) b[d] = (*bloch)[d];
    qp_ = bloch.has_value();
    const int n = (int)positions.size();
    // the point steps of the construction on the GPU for all but small systems
    const bool on_device = n > 0 && pdmkb::tree_build_on_device(n, 20000);
    p_->plan = std::make_unique<pdmkb::Plan>(
        on_device ? pdmkb::build_plan_device(c, n, pos.data(), n_digits, n_per_leaf, nz, qp_ ? b : nullptr)
                  : pdmkb::build_plan(c, n, pos.data(), n_digits, n_per_leaf, nz, qp_ ? b : nullptr));
    p_->single = std::is_same<Real, float>::value;
    p_->dev = std::make_unique<pdmkb::DeviceTree>(*p_->plan, -1, /*fp64_working_set=*/!p_->single);
    n_src_ = p_->plan->n_src;
    rc_ = p_->plan->rc;
}

template <typename Real, int DIM>
PeriodicDMKTreeT<Real, DIM>::~PeriodicDMKTreeT() = default;

template <typename Real, int DIM>
std::vector<Real> PeriodicDMKTreeT<Real, DIM>::evaluate(const std::vector<double>& charges) {
    if (qp_) throw std::logic_error("evaluate: bloch is set - use evaluate_complex()");
    EvalTiming t;
    return evaluate_timed(charges, t);
}

template <typename Real, int DIM>
std::vector<Real> PeriodicDMKTreeT<Real, DIM>::evaluate_timed(const std::vector<double>& charges, EvalTiming& timing) {
    if (qp_) throw std::logic_error("evaluate_timed: bloch is set - use evaluate_complex()");
    if ((int)charges.size() != n_src_) throw std::invalid_argument("charges size != n_src");
    std::vector<double> pot(n_src_);
    pdmkb::StageTimes st;
    if (p_->single)
        p_->dev->evaluate_multi_host(charges.data(), 1, pot.data(), /*pot_float=*/false, /*fp32=*/true, &st);
    else
        p_->dev->evaluate_host(charges.data(), pot.data(), &st);
    timing.dmk_ms = st.dmk_ms;
    timing.direct_ms = st.direct_ms;
    timing.nufft_ms = st.nufft_ms;
    timing.build_ms = 0.0;
    return std::vector<Real>(pot.begin(), pot.end());
}

template <typename Real, int DIM>
std::vector<Real> PeriodicDMKTreeT<Real, DIM>::evaluate_multi(const std::vector<double>& charges, int k) {
    if (qp_) throw std::logic_error("evaluate_multi: bloch is set - use evaluate_complex()");
    if (k <= 0 || (int64_t)charges.size() != (int64_t)n_src_ * k)
        throw std::invalid_argument("charges size != n_src * k");
    std::vector<double> pot((size_t)n_src_ * k);
    p_->dev->evaluate_multi_host(charges.data(), k, pot.data(), /*pot_float=*/false, /*fp32=*/p_->single, nullptr);
    return std::vector<Real>(pot.begin(), pot.end());
}

template <typename Real, int DIM>
std::vector<std::complex<Real>> PeriodicDMKTreeT<Real, DIM>::evaluate_complex(const std::vector<double>& charges) {
    if (!qp_) throw std::logic_error("evaluate_complex: bloch not set at construction");
    if ((int)charges.size() != n_src_) throw std::invalid_argument("charges size != n_src");
    std::vector<double> pot(2 * (size_t)n_src_);
    p_->dev->evaluate_complex_host(charges.data(), pot.data());
    std::vector<std::complex<Real>> out((size_t)n_src_);
    for (int i = 0; i < n_src_; ++i) out[i] = std::complex<Real>((Real)pot[2 * (size_t)i], (Real)pot[2 * (size_t)i + 1]);
    return out;
}

template class PeriodicDMKTreeT<double, 3>;
template class PeriodicDMKTreeT<float, 3>;

AutoPeriodicDMKTree::AutoPeriodicDMKTree(const Mat3& cell, const std::vector<Vec3>& positions, int n_digits,
                                         int n_per_leaf, int nz) {
    single_precision_ = n_digits <= 6;
    if (single_precision_)
        impl_ = std::make_unique<PeriodicDMKTreeT<float, 3>>(cell, positions, n_digits, n_per_leaf, nz);
    else
        impl_ = std::make_unique<PeriodicDMKTreeT<double, 3>>(cell, positions, n_digits, n_per_leaf, nz);
}

std::variant<std::vector<float>, std::vector<double>> AutoPeriodicDMKTree::evaluate(const std::vector<double>& charges) {
    if (single_precision_) return std::get<std::unique_ptr<PeriodicDMKTreeT<float, 3>>>(impl_)->evaluate(charges);
    return std::get<std::unique_ptr<PeriodicDMKTreeT<double, 3>>>(impl_)->evaluate(charges);
}

AutoPeriodicDMKTree make_periodic_dmk_tree(const Mat3& cell, const std::vector<Vec3>& positions, int n_digits,
                                           int n_per_leaf, int nz) {
    return AutoPeriodicDMKTree(cell, positions, n_digits, n_per_leaf, nz);
}

}  // namespace pdmk
