// extern "C" boundary of libpdmk_b200.so.  See include/pdmk/pdmk_capi.h for the
// contract; each entry cites the reference interface it replaces there.
#include "pdmk/pdmk_capi.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../device/ewald.cuh"
#include "../device/tree_build.hpp"
#include "../host/plan.hpp"
#include "batch.hpp"
#include "pdmk/campaign_ref_io.hpp"
#include "impl.hpp"
#include "pdmk/periodic_dmk.hpp"

namespace {

thread_local std::string g_last_error;

void set_error(const char* where, const char* what) {
    g_last_error = std::string(where) + ": " + what;
    std::fprintf(stderr, "%s\n", g_last_error.c_str());
}

// CUDA failures surface as std::runtime_error whose message starts with
// "CUDA error" / "cuFFT error"; they map to -2.
int fail(const char* where, const std::exception& e) {
    set_error(where, e.what());
    const std::string m = e.what();
    return (m.rfind("CUDA error", 0) == 0 || m.rfind("cuFFT error", 0) == 0) ? -2 : -1;
}

pdmk::Mat3 to_mat3(const double* c) {
    pdmk::Mat3 h;
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) h[j][i] = c[i + 3 * j];
    return h;
}

std::vector<pdmk::Vec3> to_positions(const double* p, int n) {
    std::vector<pdmk::Vec3> v(n);
    for (int i = 0; i < n; ++i) v[i] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    return v;
}

template <typename Real>
void* create_impl(const double* cell, int n, const double* pos, int nd, int npl, int nz) {
    try {
        if (!cell || !pos) throw std::invalid_argument("null cell or positions");
        if (n <= 0) throw std::invalid_argument("N must be positive");
        g_last_error.clear();
        return new pdmk::PeriodicDMKTreeT<Real, 3>(to_mat3(cell), to_positions(pos, n), nd, npl, nz);
    } catch (const std::exception& e) {
        set_error("pdmk_create", e.what());
        return nullptr;
    }
}

template <typename Real>
void* create_qp_impl(const double* cell, int n, const double* pos, int nd, int npl, int nz, const double* bloch) {
    try {
        if (!cell || !pos || !bloch) throw std::invalid_argument("null cell, positions or bloch");
        if (n <= 0) throw std::invalid_argument("N must be positive");
        g_last_error.clear();
        return new pdmk::PeriodicDMKTreeT<Real, 3>(to_mat3(cell), to_positions(pos, n), nd, npl, nz,
                                                   std::array<double, 3>{bloch[0], bloch[1], bloch[2]});
    } catch (const std::exception& e) {
        set_error("pdmk_create_qp", e.what());
        return nullptr;
    }
}

template <typename Real, typename Out>
int evaluate_complex_impl(void* h, const double* q, Out* pot2, bool device) {
    if (!h) {
        set_error("pdmk_evaluate_complex", "null handle");
        return -1;
    }
    try {
        if (!q || !pot2) throw std::invalid_argument("null charges or output");
        auto* dv = static_cast<pdmk::PeriodicDMKTreeT<Real, 3>*>(h)->impl()->dev.get();
        if (device) {
            dv->evaluate_complex_device(q, reinterpret_cast<double*>(pot2));
            PDMK_CUDA_CHECK(cudaStreamSynchronize(dv->stream()));
        } else if (std::is_same<Out, double>::value) {
            dv->evaluate_complex_host(q, reinterpret_cast<double*>(pot2));
        } else {
            std::vector<double> tmp(2 * (size_t)dv->n_points());
            dv->evaluate_complex_host(q, tmp.data());
            for (size_t i = 0; i < tmp.size(); ++i) pot2[i] = (Out)tmp[i];
        }
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_evaluate_complex", e);
    }
}

template <typename Real, typename Out>
int evaluate_impl(void* h, const double* q, Out* pot, double* timing4) {
    if (!h) {
        set_error("pdmk_evaluate", "null handle");
        return -1;
    }
    try {
        if (!q || !pot) throw std::invalid_argument("null charges or output");
        auto* t = static_cast<pdmk::PeriodicDMKTreeT<Real, 3>*>(h);
        auto* dv = t->impl()->dev.get();
        pdmkb::StageTimes st;
        // Straight from the caller's buffers: no intermediate host copies.
        if (std::is_same<Real, double>::value)
            dv->evaluate_host(q, reinterpret_cast<double*>(pot), &st);
        else
            dv->evaluate_multi_host(q, 1, pot, /*pot_float=*/std::is_same<Out, float>::value, /*fp32=*/true, &st);
        if (timing4) {
            timing4[0] = st.nufft_ms;
            timing4[1] = st.dmk_ms;
            timing4[2] = st.direct_ms;
            timing4[3] = 0.0;
        }
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_evaluate", e);
    }
}

template <typename Real, typename Out>
int evaluate_multi_impl(void* h, int k, const double* q, Out* pot) {
    if (!h) {
        set_error("pdmk_evaluate_multi", "null handle");
        return -1;
    }
    try {
        if (!q || !pot) throw std::invalid_argument("null charges or output");
        if (k <= 0) throw std::invalid_argument("k must be positive");
        auto* t = static_cast<pdmk::PeriodicDMKTreeT<Real, 3>*>(h);
        t->impl()->dev->evaluate_multi_host(q, k, pot, std::is_same<Out, float>::value,
                                            /*fp32=*/std::is_same<Real, float>::value, nullptr);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_evaluate_multi", e);
    }
}

template <typename Real>
int stage_times_impl(void* h, double* out8) {
    if (!h || !out8) {
        set_error("pdmk_stage_times", "null handle or output");
        return -1;
    }
    try {
        auto* dv = static_cast<pdmk::PeriodicDMKTreeT<Real, 3>*>(h)->impl()->dev.get();
        const pdmkb::StageTimes t = dv->last_was_multi_ ? dv->last_multi_times() : dv->last_times();
        out8[0] = t.dmk_ms;
        out8[1] = t.near_ms;
        out8[2] = t.nufft_ms;
        out8[3] = t.finalize_ms;
        out8[4] = t.dmk_ms + t.direct_ms + t.nufft_ms;
        out8[5] = (double)dv->near_pairs_culled();
        out8[6] = (double)dv->near_pairs_nominal();
        out8[7] = (double)dv->near_coeffs();
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_stage_times", e);
    }
}

template <typename Real>
int info_impl(void* h, int64_t* out) {
    if (!h || !out) {
        set_error("pdmk_info", "null handle or output");
        return -1;
    }
    auto* t = static_cast<pdmk::PeriodicDMKTreeT<Real, 3>*>(h);
    auto* im = t->impl();
    const pdmkb::Plan& P = *im->plan;
    int nlt = 0;
    for (int b = 0; b < P.nboxes; ++b)
        if (P.is_leaf[b] && P.trg_count[b] > 0) nlt++;
    out[0] = P.n_src;
    out[1] = P.n_all;
    out[2] = P.nboxes;
    out[3] = P.nlevels;
    out[4] = nlt;
    out[5] = P.p;
    out[6] = P.n_pw;
    out[7] = im->dev->launches_per_evaluate();
    out[8] = (int64_t)im->dev->device_bytes();
    out[9] = (int64_t)P.ms * P.mt * P.mu;
    out[10] = (int64_t)P.list1.size();
    out[11] = P.n_pw_exp;
    out[12] = im->dev->multi_launches_;
    out[13] = P.dp.n_digits_tree;
    out[14] = im->dev->mixed_allowed() ? 1 : 0;
    out[15] = im->dev->translate_boxes();
    return 0;
}

template <typename Real>
int multi_device_impl(void* h, int k, const double* Q, double* pot, bool fp32) {
    if (!h) {
        set_error("pdmk_evaluate_multi_device", "null handle");
        return -1;
    }
    try {
        if (!Q || !pot) throw std::invalid_argument("null device pointer");
        auto* t = static_cast<pdmk::PeriodicDMKTreeT<Real, 3>*>(h);
        auto* dv = t->impl()->dev.get();
        dv->evaluate_multi_device(Q, k, pot, fp32, nullptr);
        PDMK_CUDA_CHECK(cudaStreamSynchronize(dv->stream()));
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_evaluate_multi_device", e);
    }
}

}  // namespace

extern "C" {

const char* pdmk_last_error(void) { return g_last_error.c_str(); }

void* pdmk_create_double(const double* cell, int N, const double* pos, int nd, int npl, int nz) {
    return create_impl<double>(cell, N, pos, nd, npl, nz);
}
void* pdmk_create_float(const double* cell, int N, const double* pos, int nd, int npl, int nz) {
    return create_impl<float>(cell, N, pos, nd, npl, nz);
}
int pdmk_evaluate_double(void* h, int, const double*, const double* q, double* pot) {
    return evaluate_impl<double, double>(h, q, pot, nullptr);
}
int pdmk_evaluate_float(void* h, int, const double*, const double* q, float* pot) {
    return evaluate_impl<float, float>(h, q, pot, nullptr);
}
int pdmk_evaluate_timed_double(void* h, int, const double*, const double* q, double* pot, double* t4) {
    return evaluate_impl<double, double>(h, q, pot, t4);
}
int pdmk_evaluate_timed_float(void* h, int, const double*, const double* q, float* pot, double* t4) {
    return evaluate_impl<float, float>(h, q, pot, t4);
}
int pdmk_evaluate_multi_double(void* h, int, int k, const double* q, double* pot) {
    return evaluate_multi_impl<double, double>(h, k, q, pot);
}
int pdmk_evaluate_multi_float(void* h, int, int k, const double* q, float* pot) {
    return evaluate_multi_impl<float, float>(h, k, q, pot);
}
void* pdmk_batch_create(int nsys, const double* cells, const int* Ns, const double* pos, int nd, int npl, int nz) {
    try {
        g_last_error.clear();
        return new pdmkb::TreeBatch(nsys, cells, Ns, pos, nd, npl, nz, /*single=*/nd <= 6);
    } catch (const std::exception& e) {
        set_error("pdmk_batch_create", e.what());
        return nullptr;
    }
}
void* pdmk_batch_create_double(int nsys, const double* cells, const int* Ns, const double* pos, int nd, int npl,
                               int nz) {
    try {
        g_last_error.clear();
        return new pdmkb::TreeBatch(nsys, cells, Ns, pos, nd, npl, nz, /*single=*/false);
    } catch (const std::exception& e) {
        set_error("pdmk_batch_create_double", e.what());
        return nullptr;
    }
}
int pdmk_batch_evaluate(void* h, const double* q, double* pot) {
    if (!h) {
        set_error("pdmk_batch_evaluate", "null handle");
        return -1;
    }
    try {
        static_cast<pdmkb::TreeBatch*>(h)->evaluate(q, pot, /*pot_float=*/false);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_batch_evaluate", e);
    }
}
int pdmk_batch_evaluate_float(void* h, const double* q, float* pot) {
    if (!h) {
        set_error("pdmk_batch_evaluate_float", "null handle");
        return -1;
    }
    try {
        static_cast<pdmkb::TreeBatch*>(h)->evaluate(q, pot, /*pot_float=*/true);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_batch_evaluate_float", e);
    }
}
int pdmk_batch_info(void* h, int64_t* out4) {
    if (!h || !out4) {
        set_error("pdmk_batch_info", "null handle or output");
        return -1;
    }
    const auto* b = static_cast<pdmkb::TreeBatch*>(h);
    out4[0] = b->n_systems();
    out4[1] = b->total_points();
    out4[2] = (int64_t)b->device_bytes();
    out4[3] = b->single() ? 1 : 0;
    return 0;
}
void pdmk_batch_destroy(void* h) { delete static_cast<pdmkb::TreeBatch*>(h); }
void pdmk_destroy_double(void* h) { delete static_cast<pdmk::PeriodicDMKTreeT<double, 3>*>(h); }
void pdmk_destroy_float(void* h) { delete static_cast<pdmk::PeriodicDMKTreeT<float, 3>*>(h); }

int pdmk_evaluate_device_double(void* h, const double* q_dev, double* pot_dev) {
    if (!h) {
        set_error("pdmk_evaluate_device", "null handle");
        return -1;
    }
    try {
        if (!q_dev || !pot_dev) throw std::invalid_argument("null device pointer");
        auto* t = static_cast<pdmk::PeriodicDMKTreeT<double, 3>*>(h);
        auto* dv = t->impl()->dev.get();
        dv->evaluate_device(q_dev, pot_dev, nullptr);
        PDMK_CUDA_CHECK(cudaStreamSynchronize(dv->stream()));
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_evaluate_device", e);
    }
}

int pdmk_evaluate_device_float(void* h, const double* q_dev, float* pot_dev) {
    (void)q_dev;
    (void)pot_dev;
    if (!h) {
        set_error("pdmk_evaluate_device", "null handle");
        return -1;
    }
    set_error("pdmk_evaluate_device_float", "not available for this tree type: use pdmk_evaluate_multi_device_float");
    return -1;
}

int pdmk_evaluate_multi_device_double(void* h, int k, const double* Q_dev, double* pot_dev, int mixed) {
    return multi_device_impl<double>(h, k, Q_dev, pot_dev, mixed != 0);
}

int pdmk_evaluate_multi_device_float(void* h, int k, const double* Q_dev, double* pot_dev) {
    return multi_device_impl<float>(h, k, Q_dev, pot_dev, true);
}

int pdmk_evaluate_multi_float_qf32(void* h, int, int k, const float* q, float* pot) {
    if (!h) {
        set_error("pdmk_evaluate_multi_float_qf32", "null handle");
        return -1;
    }
    try {
        if (!q || !pot) throw std::invalid_argument("null charges or output");
        if (k <= 0) throw std::invalid_argument("k must be positive");
        auto* t = static_cast<pdmk::PeriodicDMKTreeT<float, 3>*>(h);
        t->impl()->dev->evaluate_multi_host_f32(q, k, pot, /*fp32=*/true);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_evaluate_multi_float_qf32", e);
    }
}

int pdmk_evaluate_multi_device_float_qf32(void* h, int k, const float* Q_dev, double* pot_dev) {
    if (!h) {
        set_error("pdmk_evaluate_multi_device_float_qf32", "null handle");
        return -1;
    }
    try {
        if (!Q_dev || !pot_dev) throw std::invalid_argument("null device pointer");
        auto* t = static_cast<pdmk::PeriodicDMKTreeT<float, 3>*>(h);
        auto* dv = t->impl()->dev.get();
        dv->evaluate_multi_device_f32(Q_dev, k, pot_dev, /*fp32=*/true, nullptr);
        PDMK_CUDA_CHECK(cudaStreamSynchronize(dv->stream()));
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_evaluate_multi_device_float_qf32", e);
    }
}

int pdmk_evaluate_grad_double(void* h, int, const double*, const double* q, double* pot, double* grad) {
    if (!h) {
        set_error("pdmk_evaluate_grad_double", "null handle");
        return -1;
    }
    try {
        if (!q || !pot || !grad) throw std::invalid_argument("null charges or output");
        auto* t = static_cast<pdmk::PeriodicDMKTreeT<double, 3>*>(h);
        t->impl()->dev->evaluate_grad_host(q, pot, grad);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_evaluate_grad_double", e);
    }
}

int pdmk_evaluate_grad_device_double(void* h, const double* q_dev, double* pot_dev, double* grad_dev) {
    if (!h) {
        set_error("pdmk_evaluate_grad_device_double", "null handle");
        return -1;
    }
    try {
        if (!q_dev || !pot_dev || !grad_dev) throw std::invalid_argument("null device pointer");
        auto* t = static_cast<pdmk::PeriodicDMKTreeT<double, 3>*>(h);
        t->impl()->dev->evaluate_grad_device(q_dev, pot_dev, grad_dev);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_evaluate_grad_device_double", e);
    }
}

void* pdmk_create_qp_double(const double* cell, int N, const double* pos, int nd, int npl, int nz,
                            const double* bloch) {
    return create_qp_impl<double>(cell, N, pos, nd, npl, nz, bloch);
}
void* pdmk_create_qp_float(const double* cell, int N, const double* pos, int nd, int npl, int nz,
                           const double* bloch) {
    return create_qp_impl<float>(cell, N, pos, nd, npl, nz, bloch);
}
int pdmk_evaluate_complex_double(void* h, int, const double*, const double* q, double* pot2) {
    return evaluate_complex_impl<double, double>(h, q, pot2, false);
}
int pdmk_evaluate_complex_float(void* h, int, const double*, const double* q, float* pot2) {
    return evaluate_complex_impl<float, float>(h, q, pot2, false);
}
int pdmk_evaluate_complex_device_double(void* h, const double* q_dev, double* pot2_dev) {
    return evaluate_complex_impl<double, double>(h, q_dev, pot2_dev, true);
}

int pdmk_evaluate_parts_double(void* h, const double* q, double* tree_part, double* far_part) {
    if (!h) {
        set_error("pdmk_evaluate_parts", "null handle");
        return -1;
    }
    try {
        if (!q || !tree_part || !far_part) throw std::invalid_argument("null buffer");
        auto* t = static_cast<pdmk::PeriodicDMKTreeT<double, 3>*>(h);
        t->impl()->dev->evaluate_parts_host(q, tree_part, far_part);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_evaluate_parts", e);
    }
}

int pdmk_evaluate_device_noalloc_double(void* h, const double* q_dev, double* pot_dev) {
    if (!h) {
        set_error("pdmk_evaluate_device_noalloc_double", "null handle");
        return -1;
    }
    try {
        if (!q_dev || !pot_dev) throw std::invalid_argument("null device pointer");
        auto* t = static_cast<pdmk::PeriodicDMKTreeT<double, 3>*>(h);
        t->impl()->dev->evaluate_device_noalloc(q_dev, pot_dev);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_evaluate_device_noalloc_double", e);
    }
}

int pdmk_sha256(const void* data, uint64_t len, unsigned char* out32) {
    if ((!data && len) || !out32) {
        set_error("pdmk_sha256", "null buffer");
        return -1;
    }
    pdmk::campaign::sha256(static_cast<const uint8_t*>(data), (size_t)len, out32);
    return 0;
}

int pdmk_campaign_write(const char* path, uint32_t config_id, uint32_t digits, uint32_t prec, uint64_t seed,
                        const double* cell9, uint32_t N, const double* pos, const double* chg, uint32_t M,
                        const uint32_t* ref_idx, const double* ref_u) {
    try {
        if (!path || !cell9 || (N && (!pos || !chg)) || (M && (!ref_idx || !ref_u)))
            throw std::invalid_argument("null argument");
        if (digits > 255 || prec > 255) throw std::invalid_argument("digits and prec must fit one byte");
        pdmk::campaign::RefData d{};
        d.header.config_id = config_id;
        d.header.N = N;
        d.header.digits = (uint8_t)digits;
        d.header.prec = (uint8_t)prec;
        d.header.seed = seed;
        std::memcpy(d.cell, cell9, sizeof(d.cell));
        d.ref_idx.assign(ref_idx, ref_idx + M);
        d.ref_u.assign(ref_u, ref_u + M);
        d.pos.assign(pos, pos + 3 * (size_t)N);
        d.chg.assign(chg, chg + N);
        pdmk::campaign::write_ref(path, d);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_campaign_write", e);
    }
}

int pdmk_campaign_read_header(const char* path, uint32_t* out5, uint64_t* seed) {
    try {
        if (!path || !out5) throw std::invalid_argument("null argument");
        const pdmk::campaign::RefData d = pdmk::campaign::read_ref(path);
        out5[0] = d.header.config_id;
        out5[1] = d.header.N;
        out5[2] = d.header.M;
        out5[3] = d.header.digits;
        out5[4] = d.header.prec;
        if (seed) *seed = d.header.seed;
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_campaign_read_header", e);
    }
}

int pdmk_campaign_read(const char* path, double* cell9, double* pos, double* chg, uint32_t* ref_idx, double* ref_u) {
    try {
        if (!path || !cell9 || !pos || !chg || !ref_idx || !ref_u) throw std::invalid_argument("null argument");
        const pdmk::campaign::RefData d = pdmk::campaign::read_ref(path);
        std::memcpy(cell9, d.cell, sizeof(d.cell));
        std::copy(d.pos.begin(), d.pos.end(), pos);
        std::copy(d.chg.begin(), d.chg.end(), chg);
        std::copy(d.ref_idx.begin(), d.ref_idx.end(), ref_idx);
        std::copy(d.ref_u.begin(), d.ref_u.end(), ref_u);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_campaign_read", e);
    }
}

int pdmk_plan_digest(const double* cell, int N, const double* pos, int n_digits, int n_per_leaf, int nz,
                     int on_device, unsigned char* out32, double* build_ms) {
    try {
        if (!cell || !pos || !out32) throw std::invalid_argument("null argument");
        if (N <= 0) throw std::invalid_argument("N must be positive");
        const auto t0 = std::chrono::steady_clock::now();
        const pdmkb::Plan P = on_device ? pdmkb::build_plan_device(cell, N, pos, n_digits, n_per_leaf, nz)
                                        : pdmkb::build_plan(cell, N, pos, n_digits, n_per_leaf, nz);
        const auto t1 = std::chrono::steady_clock::now();
        if (build_ms) *build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        std::vector<uint8_t> b;
        auto put = [&](const void* p, size_t n) {
            const uint8_t* c = static_cast<const uint8_t*>(p);
            b.insert(b.end(), c, c + n);
        };
        auto vec = [&](const auto& v) { put(v.data(), v.size() * sizeof(v[0])); };
        const int64_t head[3] = {P.n_all, P.nboxes, P.nlevels};
        put(head, sizeof(head));
        vec(P.src_sorted); vec(P.trg_sorted); vec(P.src_perm); vec(P.trg_perm); vec(P.src_charge_idx);
        vec(P.img_src_idx); vec(P.depth); vec(P.parent); vec(P.nchild); vec(P.children); vec(P.colleagues);
        vec(P.centers); vec(P.src_start); vec(P.src_count); vec(P.trg_start); vec(P.trg_count);
        vec(P.list1_start); vec(P.list1); vec(P.ifpwexp); vec(P.iftensprodeval); vec(P.has_proxy_from_children);
        vec(P.direct_work);
        pdmk::campaign::sha256(b.data(), b.size(), out32);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_plan_digest", e);
    }
}

int pdmk_info_double(void* h, int64_t* out) { return info_impl<double>(h, out); }

int pdmk_stage_times_double(void* h, double* out8) { return stage_times_impl<double>(h, out8); }
int pdmk_stage_times_float(void* h, double* out8) { return stage_times_impl<float>(h, out8); }

int pdmk_fma_peak(int fp64, double* tflops) {
    try {
        if (!tflops) throw std::invalid_argument("null output");
        *tflops = pdmkb::dev::fma_probe_tflops(fp64 != 0);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_fma_peak", e);
    }
}
int pdmk_tc_peak(int kind, double* tflops) {
    try {
        if (!tflops) throw std::invalid_argument("null output");
        *tflops = pdmkb::dev::tc_probe_tflops(kind);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_tc_peak", e);
    }
}
int pdmk_info_float(void* h, int64_t* out) { return info_impl<float>(h, out); }

// ---------------------------------------------------------------------------
// Ewald summation on the GPU (csrc/device/ewald.cu): cell-list real-space sum
// within r_cut = s/alpha, NUFFT reciprocal sum over |k| <= 2 s alpha, self term
// -2 alpha/sqrt(pi) q_i and the charged-system energy correction.
// ---------------------------------------------------------------------------
int pdmk_ewald_nufft(const double* cell, int N, const double* pos, const double* q, double s, double* pot,
                     double* energy) {
    try {
        if (!cell || !pos || !q || !pot) throw std::invalid_argument("null buffer");
        pdmkb::ewald_gpu(cell, N, pos, q, s, pot, energy);
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_ewald_nufft", e);
    }
}

// ---------------------------------------------------------------------------
// Cubic cover: frame from the two longest lattice vectors, cube side from the
// rotated bounding box's shortest width split into nz layers.
// ---------------------------------------------------------------------------
int pdmk_optimize_cubic_cover(const double* cell, int nz, int* m_out, int* n_out, int* p_out, double* e1_out,
                              double* e2_out, double* e3_out, double* s_out, double* cost_out) {
    try {
        if (nz <= 0) return 1;
        if (!cell || !m_out || !n_out || !p_out || !e1_out || !e2_out || !e3_out || !s_out || !cost_out)
            throw std::invalid_argument("null buffer");
        const double* a[3] = {cell, cell + 3, cell + 6};
        auto dot = [](const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
        double nrm[3];
        for (int d = 0; d < 3; ++d) nrm[d] = std::sqrt(dot(a[d], a[d]));
        int idx[3] = {0, 1, 2};
        if (nrm[idx[0]] < nrm[idx[1]]) std::swap(idx[0], idx[1]);
        if (nrm[idx[1]] < nrm[idx[2]]) std::swap(idx[1], idx[2]);
        if (nrm[idx[0]] < nrm[idx[1]]) std::swap(idx[0], idx[1]);
        const double* b1 = a[idx[0]];
        const double* b2 = a[idx[1]];
        if (!(nrm[idx[0]] > 0)) throw std::invalid_argument("degenerate lattice (zero-norm vector)");
        double e1[3], e2[3], e3[3];
        for (int d = 0; d < 3; ++d) e1[d] = b1[d] / nrm[idx[0]];
        const double p12 = dot(b2, e1);
        double v2[3];
        for (int d = 0; d < 3; ++d) v2[d] = b2[d] - p12 * e1[d];
        const double nv2 = std::sqrt(dot(v2, v2));
        if (!(nv2 > 0)) throw std::invalid_argument("degenerate lattice (parallel vectors)");
        for (int d = 0; d < 3; ++d) e2[d] = v2[d] / nv2;
        e3[0] = e1[1] * e2[2] - e1[2] * e2[1];
        e3[1] = e1[2] * e2[0] - e1[0] * e2[2];
        e3[2] = e1[0] * e2[1] - e1[1] * e2[0];
        double W[3] = {0, 0, 0};
        for (int d = 0; d < 3; ++d) {
            W[0] += std::fabs(dot(a[d], e1));
            W[1] += std::fabs(dot(a[d], e2));
            W[2] += std::fabs(dot(a[d], e3));
        }
        const double s = W[2] / nz;
        const int m = std::max(1, (int)std::ceil(W[0] / s)), n = std::max(1, (int)std::ceil(W[1] / s));
        double c[3] = {a[1][1] * a[2][2] - a[1][2] * a[2][1], a[1][2] * a[2][0] - a[1][0] * a[2][2],
                       a[1][0] * a[2][1] - a[1][1] * a[2][0]};
        const double V = std::fabs(dot(a[0], c));
        *m_out = m;
        *n_out = n;
        *p_out = nz;
        for (int d = 0; d < 3; ++d) {
            e1_out[d] = e1[d];
            e2_out[d] = e2[d];
            e3_out[d] = e3[d];
        }
        *s_out = s;
        *cost_out = (double)((m + 2) * (n + 2) * (nz + 2)) * s * s * s / V;
        return 0;
    } catch (const std::exception& e) {
        return fail("pdmk_optimize_cubic_cover", e);
    }
}

}  // extern "C"
