// Compiled C++ check of the public C++ API (include/pdmk/periodic_dmk.hpp)
// against the C ABI (include/pdmk/pdmk_capi.h), both from libpdmk_b200.so.
// Built by tests/test_cpp_api.py; run on a GPU it prints one line per check
// and exits non-zero on a mismatch.  The reference's own tests of this API
// (cpp/tests/test_periodic_dmk_tree.cpp:30-52, test_evaluate_timed.cpp:34-67)
// check repeatability, timing fields and evaluate_timed == evaluate.
#include <cmath>
#include <cstdio>
#include <random>
#include <stdexcept>
#include <variant>
#include <vector>

#include "pdmk/pdmk_capi.h"
#include "pdmk/periodic_dmk.hpp"

static double rel_l2(const std::vector<double>& a, const std::vector<double>& b) {
    double num = 0, den = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        num += (a[i] - b[i]) * (a[i] - b[i]);
        den += b[i] * b[i];
    }
    return std::sqrt(num / den);
}

template <typename T>
static std::vector<double> to_double(const std::vector<T>& v) {
    return std::vector<double>(v.begin(), v.end());
}

int main() {
    const int n = 3000;
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    pdmk::Mat3 cell{};  // cell[j][i] = component i of lattice vector j
    cell[0] = {1.0, 0.0, 0.0};
    cell[1] = {0.3, 0.9, 0.0};
    cell[2] = {0.2, 0.25, 0.85};
    std::vector<pdmk::Vec3> pos(n);
    std::vector<double> q(n), pos3(3 * n), cell9(9);
    double mean = 0;
    for (int i = 0; i < n; ++i) {
        const double f[3] = {U(rng), U(rng), U(rng)};
        for (int d = 0; d < 3; ++d) pos[i][d] = f[0] * cell[0][d] + f[1] * cell[1][d] + f[2] * cell[2][d];
        q[i] = 2 * U(rng) - 1;
        mean += q[i] / n;
    }
    for (int i = 0; i < n; ++i) {
        q[i] -= mean;
        for (int d = 0; d < 3; ++d) pos3[3 * i + d] = pos[i][d];
    }
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) cell9[i + 3 * j] = cell[j][i];
    int fails = 0;
    auto check = [&](const char* what, bool ok, double v) {
        std::printf("%s %s %.3e\n", ok ? "ok  " : "FAIL", what, v);
        if (!ok) ++fails;
    };

    // double tree vs the C ABI double path (same device code, same arithmetic)
    pdmk::PeriodicDMKTreeT<double, 3> td(cell, pos, 9, 40, 4);
    const std::vector<double> ud = td.evaluate(q);
    void* h = pdmk_create_double(cell9.data(), n, pos3.data(), 9, 40, 4);
    std::vector<double> uc(n);
    check("capi_create_double", h != nullptr, 0);
    check("capi_evaluate_double", pdmk_evaluate_double(h, n, pos3.data(), q.data(), uc.data()) == 0, 0);
    check("cxx_double_equals_capi", rel_l2(ud, uc) < 1e-13, rel_l2(ud, uc));
    pdmk::EvalTiming tm;
    const std::vector<double> ut = td.evaluate_timed(q, tm);
    check("evaluate_timed_equals_evaluate", rel_l2(ut, ud) < 1e-12, rel_l2(ut, ud));
    check("timing_fields_positive", tm.dmk_ms > 0 && tm.direct_ms > 0 && tm.nufft_ms > 0, tm.dmk_ms);
    check("n_points", td.n_points() == n, td.n_points());
    check("cube_size", std::abs(td.cube_size() - 0.85 / 4) < 1e-12, td.cube_size());
    pdmk_destroy_double(h);

    // float tree vs the C ABI float path, and vs the double tree (mixed precision)
    pdmk::PeriodicDMKTreeT<float, 3> tf(cell, pos, 6, 40, 4);
    const std::vector<float> uf = tf.evaluate(q);
    void* hf = pdmk_create_float(cell9.data(), n, pos3.data(), 6, 40, 4);
    std::vector<float> ucf(n);
    check("capi_evaluate_float", hf && pdmk_evaluate_float(hf, n, pos3.data(), q.data(), ucf.data()) == 0, 0);
    check("cxx_float_equals_capi", rel_l2(to_double(uf), to_double(ucf)) < 1e-7,
          rel_l2(to_double(uf), to_double(ucf)));
    pdmk::PeriodicDMKTreeT<double, 3> td6(cell, pos, 6, 40, 4);
    const std::vector<double> ud6 = td6.evaluate(q);
    check("float_tree_vs_double_tree", rel_l2(to_double(uf), ud6) < 1e-6, rel_l2(to_double(uf), ud6));
    pdmk_destroy_float(hf);

    // automatic selection: float at <= 6 digits, double above
    pdmk::AutoPeriodicDMKTree a6 = pdmk::make_periodic_dmk_tree(cell, pos, 6, 40, 4);
    pdmk::AutoPeriodicDMKTree a9 = pdmk::make_periodic_dmk_tree(cell, pos, 9, 40, 4);
    check("auto_6_is_float", a6.is_single_precision(), 0);
    check("auto_9_is_double", !a9.is_single_precision(), 0);
    auto v6 = a6.evaluate(q);
    auto v9 = a9.evaluate(q);
    check("auto_6_returns_float", std::holds_alternative<std::vector<float>>(v6), 0);
    check("auto_9_returns_double", std::holds_alternative<std::vector<double>>(v9), 0);
    if (std::holds_alternative<std::vector<float>>(v6))
        check("auto_6_equals_float_tree", rel_l2(to_double(std::get<std::vector<float>>(v6)), to_double(uf)) < 1e-7,
              rel_l2(to_double(std::get<std::vector<float>>(v6)), to_double(uf)));
    if (std::holds_alternative<std::vector<double>>(v9))
        check("auto_9_equals_double_tree", rel_l2(std::get<std::vector<double>>(v9), ud) < 1e-13,
              rel_l2(std::get<std::vector<double>>(v9), ud));

    // errors: wrong charge count throws std::invalid_argument
    bool threw = false;
    try {
        std::vector<double> bad(n - 1, 0.0);
        td.evaluate(bad);
    } catch (const std::invalid_argument&) {
        threw = true;
    }
    check("wrong_size_throws", threw, 0);
    std::printf("%d failures\n", fails);
    return fails == 0 ? 0 : 1;
}
