// DeviceTree: one-time upload of a host Plan and the evaluate pipeline.
//
// Device memory layout (all resident for the lifetime of the tree):
//   src          double4[n_all]  sorted sources (x, y, z, q); q refreshed per evaluate
//   trg          double4[N]      sorted targets (x, y, z, w0 of the target's leaf)
//   proxy_up     double[n_up * p^3]   upward Chebyshev proxy charges, (p,p,p) x fastest
//   proxy_down   double[n_down * p^3] downward proxy potentials
//   pw_out       complex[n_pw * n*n*n2] outgoing plane-wave expansions
//   tables       per level: poly2pw (n x p), poly2pw_half (n2 x p), pw2poly^T (p x n),
//                weighted pw2poly^T (p x n2), 27 fused shift stencils; c2p / p2c (8 x 3 x p x p)
//   far field    real fine grid n1*n2*n3, half spectrum n1*n2*(n3/2+1), multiplier
// Every index list is built and bounds-checked here, on the host.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <stdexcept>

#include "../host/pswf.hpp"
#include "device_tree.hpp"
#include "dmma.cuh"
#include "grad.cuh"
#include "pw_fused.cuh"
#include "sep3.cuh"
#include "tc_kernels.cuh"

namespace pdmkb {

using dev::cd;

namespace {

void check(bool ok, const char* what) {
    if (!ok) throw std::runtime_error(std::string("DeviceTree: inconsistent plan: ") + what);
}

int nice_fft_size(int n) {
    for (int m = std::max(2, n);; ++m) {
        if (m % 2) continue;
        int r = m;
        for (int f : {2, 3, 5, 7})
            while (r % f == 0) r /= f;
        if (r == 1) return m;
    }
}

#define CUFFT_CHECK(expr)                                                                      \
    do {                                                                                       \
        cufftResult _r = (expr);                                                               \
        if (_r != CUFFT_SUCCESS)                                                               \
            throw std::runtime_error("cuFFT error " + std::to_string((int)_r) + " at " #expr); \
    } while (0)

}  // namespace

template <typename T>
T* DeviceTree::alloc(size_t n) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    PDMK_CUDA_CHECK(cudaMalloc(&p, bytes));
    allocs_.push_back(p);
    bytes_ += bytes;
    return static_cast<T*>(p);
}

template <typename T>
T* DeviceTree::upload(const std::vector<T>& v) {
    T* p = alloc<T>(v.size());
    if (!v.empty()) PDMK_CUDA_CHECK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return p;
}

DeviceTree::DeviceTree(const Plan& P, int device, bool fp64_working_set) {
    try {
        init(P, device, fp64_working_set);
    } catch (...) {
        release();
        throw;
    }
}

void DeviceTree::init(const Plan& P, int device, bool fp64_working_set) {
    // PDMK_BUILD_PROFILE=1: host milliseconds of every phase below, on stderr
    const bool prof = std::getenv("PDMK_BUILD_PROFILE") != nullptr;
    auto t_prev = std::chrono::steady_clock::now();
    const char* cur = "setup";
    auto phase = [&](const char* next) {  // closes the current phase, opens the next
        if (prof) {
            const auto t = std::chrono::steady_clock::now();
            std::fprintf(stderr, "device tree %-24s %9.2f ms\n", cur,
                         std::chrono::duration<double, std::milli>(t - t_prev).count());
            t_prev = t;
        }
        cur = next;
    };
    if (device < 0) PDMK_CUDA_CHECK(cudaGetDevice(&device));
    device_ = device;
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    PDMK_CUDA_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    for (auto& e : ev_) PDMK_CUDA_CHECK(cudaEventCreate(&e));

    if (const char* tm = std::getenv("PDMK_TC_MASK")) tc_mask_ = std::atoi(tm) & 15;
    if (const char* dm = std::getenv("PDMK_FP64_DMMA")) fp64_dmma_ = std::atoi(dm) != 0;
    if (const char* mm = std::getenv("PDMK_MOMENTS_DMMA")) moments_dmma_ = std::atoi(mm) != 0;
    if (const char* ov = std::getenv("PDMK_E2E_OVERLAP")) overlap_h2d_ = std::atoi(ov) != 0;
    n_ = P.n_src;
    n_digits_ = P.dp.n_digits_tree;
    n_all_ = P.n_all;
    p_ = P.p;
    npw_ = P.n_pw;
    npw2_ = P.n_pw2;
    M_ = P.n_modes;
    const int p = p_, n = npw_, n2 = npw2_, M = M_;
    const int64_t ncoef = (int64_t)p * p * p;

    phase("far-field bins");
    // ------------------------------------------------------------------ far-field bins
    // NUFFT bins are contiguous ranges of sorted targets inside one leaf.  A leaf
    // whose subgrid would be wider than kMaxEx cells is split by grid blocks,
    // which permutes targets only inside that leaf (every stage is invariant
    // to the order of points within a leaf).
    const double eps = P.dp.eps;
    int W = (int)std::ceil(-std::log10(eps / 4.0)) + 1;
    W = std::min(14, std::max(4, W));
    const int ng[3] = {nice_fft_size(std::max(2 * P.ms, 2 * W)), nice_fft_size(std::max(2 * P.mt, 2 * W)),
                       nice_fft_size(std::max(2 * P.mu, 2 * W))};
    constexpr int kMaxEx = 48;
    std::vector<double> trg_sorted = P.trg_sorted;
    std::vector<int> trg_perm = P.trg_perm;
    std::vector<double> trg_selfw(n_, 0.0);
    std::vector<double4> pt_t(n_);
    std::vector<int4> pt_l0(n_);
    struct Bin {
        int start, count;
        int4 org, ext;
    };
    std::vector<Bin> bins;
    {
        const double* v = P.umatinv;
        auto frac_t = [&](const double* r, double* t) {
            const double s[3] = {v[0] * r[0] + v[3] * r[1] + v[6] * r[2], v[4] * r[1] + v[7] * r[2], v[8] * r[2]};
            for (int d = 0; d < 3; ++d) t[d] = (s[d] - std::floor(s[d])) * ng[d];
        };
        for (int b = 0; b < P.nboxes; ++b) {
            if (!P.is_leaf[b] || P.trg_count[b] == 0) continue;
            const int t0 = P.trg_start[b], nt = P.trg_count[b];
            check(t0 >= 0 && t0 + nt <= n_, "target range");
            const double w0 = P.w0[P.depth[b] + P.ifpwexp[b]];
            std::vector<std::array<double, 3>> tt(nt);
            for (int i = 0; i < nt; ++i) frac_t(&trg_sorted[3 * (size_t)(t0 + i)], tt[i].data());
            // unwrap each axis so the leaf's points are contiguous in grid space
            for (int d = 0; d < 3; ++d) {
                double lo = 1e300, hi = -1e300;
                for (auto& x : tt) lo = std::min(lo, x[d]), hi = std::max(hi, x[d]);
                if (hi - lo > 0.5 * ng[d])
                    for (auto& x : tt)
                        if (x[d] > 0.5 * ng[d]) x[d] -= ng[d];
            }
            std::vector<std::array<int, 3>> l0(nt);
            int lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
            for (int i = 0; i < nt; ++i)
                for (int d = 0; d < 3; ++d) {
                    l0[i][d] = (int)std::ceil(tt[i][d] - 0.5 * W);
                    lo[d] = std::min(lo[d], l0[i][d]);
                    hi[d] = std::max(hi[d], l0[i][d]);
                }
            std::vector<int> order(nt);
            std::iota(order.begin(), order.end(), 0);
            std::vector<int64_t> key(nt, 0);
            const bool split = (hi[0] - lo[0] + W > kMaxEx) || (hi[1] - lo[1] + W > kMaxEx) || (hi[2] - lo[2] + W > kMaxEx);
            if (split) {
                const int B = kMaxEx - W;
                for (int i = 0; i < nt; ++i) {
                    int64_t kx = (l0[i][0] - lo[0]) / B, ky = (l0[i][1] - lo[1]) / B, kz = (l0[i][2] - lo[2]) / B;
                    key[i] = (kx * 4096 + ky) * 4096 + kz;
                }
            }
            if (split) std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return key[a] < key[c]; });
            // apply the within-leaf permutation
            std::vector<double> pos_tmp(3 * (size_t)nt);
            std::vector<int> perm_tmp(nt);
            for (int i = 0; i < nt; ++i) {
                const int o = order[i];
                for (int d = 0; d < 3; ++d) pos_tmp[3 * i + d] = P.trg_sorted[3 * (size_t)(t0 + o) + d];
                perm_tmp[i] = P.trg_perm[t0 + o];
            }
            for (int i = 0; i < nt; ++i) {
                for (int d = 0; d < 3; ++d) trg_sorted[3 * (size_t)(t0 + i) + d] = pos_tmp[3 * i + d];
                trg_perm[t0 + i] = perm_tmp[i];
                trg_selfw[t0 + i] = w0;
                const int o = order[i];
                pt_t[t0 + i] = make_double4(tt[o][0], tt[o][1], tt[o][2], 0.0);
                pt_l0[t0 + i] = make_int4(l0[o][0], l0[o][1], l0[o][2], 0);
            }
            for (int i = 0; i < nt;) {
                int j = i;
                while (j < nt && key[order[j]] == key[order[i]]) ++j;
                Bin bn{t0 + i, j - i, make_int4(INT32_MAX, INT32_MAX, INT32_MAX, 0), make_int4(0, 0, 0, 0)};
                int bhi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
                for (int k = i; k < j; ++k) {
                    const int4 l = pt_l0[t0 + k];
                    bn.org.x = std::min(bn.org.x, l.x);
                    bn.org.y = std::min(bn.org.y, l.y);
                    bn.org.z = std::min(bn.org.z, l.z);
                    bhi[0] = std::max(bhi[0], l.x);
                    bhi[1] = std::max(bhi[1], l.y);
                    bhi[2] = std::max(bhi[2], l.z);
                }
                bn.ext = make_int4(bhi[0] - bn.org.x + W, bhi[1] - bn.org.y + W, bhi[2] - bn.org.z + W, 0);
                check(bn.ext.x <= kMaxEx && bn.ext.y <= kMaxEx && bn.ext.z <= kMaxEx, "NUFFT bin extent");
                bins.push_back(bn);
                i = j;
            }
        }
    }

    phase("points");
    // ------------------------------------------------------------------ points
    {
        std::vector<double4> src(n_all_);
        for (int i = 0; i < n_all_; ++i)
            src[i] = make_double4(P.src_sorted[3 * (size_t)i], P.src_sorted[3 * (size_t)i + 1],
                                  P.src_sorted[3 * (size_t)i + 2], 0.0);
        for (int i : P.src_charge_idx) check(i >= 0 && i < n_, "source charge index");
        src_ = upload(src);
        src_charge_idx_ = upload(P.src_charge_idx);
        std::vector<double4> trg(n_);
        for (int i = 0; i < n_; ++i)
            trg[i] = make_double4(trg_sorted[3 * (size_t)i], trg_sorted[3 * (size_t)i + 1], trg_sorted[3 * (size_t)i + 2],
                                  trg_selfw[i]);
        for (int i : trg_perm) check(i >= 0 && i < n_, "target permutation");
        trg_ = upload(trg);
        trg_perm_ = upload(trg_perm);
        pot_sorted_ = alloc<double>(n_);
        far_sorted_ = alloc<double>(n_);
        q_sorted_ = alloc<double>(n_);
        q_dev_ = alloc<double>(n_);
        pot_dev_ = alloc<double>(n_);
    }

    phase("expansions");
    // ------------------------------------------------------------------ expansions
    // Storage only for expansions that some evaluation reads.  The plan (like
    // the reference, cpp/src/dmk/pbc_tree.cpp:983-994 and its outgoing pass)
    // gives every box with points an outgoing plane-wave expansion and
    // downward coefficients; most of those boxes hold only lattice images and
    // no target, and their expansions are never read.  Read are:
    //   * plane waves of the boxes that receive incoming expansions (boxes
    //     with targets) and of their colleagues in the shift lists;
    //   * proxy_up of those boxes and of every box whose child-to-parent
    //     translation feeds one of them;
    //   * proxy_down of the boxes that receive incoming expansions or
    //     evaluate at their targets.
    // Skipping the rest changes no arithmetic on the expansions that are read.
    std::vector<int64_t> up_slot(P.nboxes, -1), down_slot(P.nboxes, -1), pw_slot(P.nboxes, -1);
    std::vector<char> incoming(P.nboxes, 0), leaf_eval(P.nboxes, 0);
    // Image boxes that are exact lattice translates of an original box of the
    // same level: every source is the image of a source of that box under one
    // lattice vector D, the counts agree and the centres differ by D.  Proxy
    // moments and outgoing expansions are taken about the box centre, so such
    // a box shares the original's (they differ only by the rounding of the
    // image positions); it gets no storage and no work of its own.  With a
    // cell whose lattice vectors are multiples of the box size (cubes) this
    // covers every image-only box; triclinic images straddle boxes and none
    // qualify.  Quasi-periodic trees share nothing: an image box's charges
    // carry the Bloch phase of its lattice vector.
    std::vector<int> alias(P.nboxes, -1);
    if (!P.qp) {
        std::vector<int> orig_of(n_, -1);
        std::vector<double> disp(3 * (size_t)n_all_);
        std::vector<char> is_orig(n_all_, 0);
        for (int s = 0; s < n_all_; ++s) {
            const int q = P.src_charge_idx[s];
            double m = 0.0;
            for (int d = 0; d < 3; ++d) {
                disp[3 * (size_t)s + d] = P.src_sorted[3 * (size_t)s + d] - P.r_user[3 * (size_t)q + d];
                m = std::max(m, std::abs(disp[3 * (size_t)s + d]));
            }
            if (m <= 1e-12) {
                is_orig[s] = 1;
                orig_of[q] = s;
            }
        }
        std::vector<int> box_at(n_all_, -1);
        for (int l = 0; l < P.nlevels; ++l) {
            for (int b : P.level_boxes[l])
                for (int s = P.src_start[b]; s < P.src_start[b] + P.src_count[b]; ++s) box_at[s] = b;
            for (int b : P.level_boxes[l]) {
                const int s0 = P.src_start[b], ns = P.src_count[b];
                if (ns <= 0) continue;
                const double* D = &disp[3 * (size_t)s0];
                bool ok = !is_orig[s0];
                const int o0 = orig_of[P.src_charge_idx[s0]];
                const int B = o0 >= 0 ? box_at[o0] : -1;
                ok = ok && B >= 0 && B != b && P.depth[B] == l && P.src_count[B] == ns;
                for (int s = s0; s < s0 + ns && ok; ++s) {
                    const int o = orig_of[P.src_charge_idx[s]];
                    ok = !is_orig[s] && o >= 0 && box_at[o] == B;
                    for (int d = 0; d < 3 && ok; ++d)
                        ok = std::abs(disp[3 * (size_t)s + d] - D[d]) <= 1e-9 * (1.0 + std::abs(D[d]));
                }
                for (int d = 0; d < 3 && ok; ++d)
                    ok = std::abs(P.centers[3 * b + d] - P.centers[3 * B + d] - D[d]) <= 1e-9 * (1.0 + std::abs(D[d]));
                if (ok) alias[b] = B;
            }
            // box_at of this level's sources is overwritten by the next level
            for (int b : P.level_boxes[l])
                for (int s = P.src_start[b]; s < P.src_start[b] + P.src_count[b]; ++s) box_at[s] = -1;
        }
        for (int b = 0; b < P.nboxes; ++b) n_alias_ += alias[b] >= 0;
    }
    {
        std::vector<char> need_pw(P.nboxes, 0), need_up(P.nboxes, 0);
        for (int b = 0; b < P.nboxes; ++b) {
            incoming[b] = P.ifpwexp[b] && P.src_count[b] + P.trg_count[b] > 0 && P.trg_count[b] > 0;
            leaf_eval[b] = P.iftensprodeval[b] && P.trg_count[b] > 0;
            if (incoming[b]) check(P.pw_off[b] >= 0 && P.proxy_down_off[b] >= 0, "form-eval box storage");
            if (leaf_eval[b]) check(P.proxy_down_off[b] >= 0, "leaf proxy_down");
        }
        for (int b = 0; b < P.nboxes; ++b) {
            if (!incoming[b]) continue;
            need_pw[b] = 1;
            for (int ind = 0; ind < 27; ++ind) {
                const int nb = P.colleagues[b][ind];
                if (nb < 0 || nb == b || (P.is_leaf[b] && P.is_leaf[nb]) || P.pw_off[nb] < 0) continue;
                need_pw[nb] = 1;
            }
        }
        // a translate's plane waves are its original's
        for (int b = 0; b < P.nboxes; ++b)
            if (need_pw[b] && alias[b] >= 0) need_pw[alias[b]] = 1;
        // top-down: a box's proxy_up is read by its own outgoing transform or
        // through the translation into a parent whose proxy_up is read (and
        // formed here: a translate parent borrows its original's)
        for (int l = 0; l < P.nlevels; ++l) {
            for (int b : P.level_boxes[l]) {
                const int par = P.parent[b];
                const bool via = par >= 0 && need_up[par] && alias[par] < 0 && P.has_proxy_from_children[par] &&
                                 P.src_count[b] > 0 && P.ifpwexp[b];
                need_up[b] = need_pw[b] || via;
            }
            for (int b : P.level_boxes[l])
                if (need_up[b] && alias[b] >= 0) need_up[alias[b]] = 1;
            for (int b : P.level_boxes[l])
                if (need_up[b]) check(P.proxy_up_off[b] >= 0, "proxy_up storage");
        }
        for (int l = 0; l < P.nlevels; ++l) {
            for (int b : P.level_boxes[l]) {
                if (alias[b] >= 0) continue;
                if (need_up[b]) up_slot[b] = n_up_++;
                if (need_pw[b]) pw_slot[b] = n_pw_++;
            }
            for (int b : P.level_boxes[l]) {
                if (alias[b] < 0) continue;
                if (need_up[b]) up_slot[b] = up_slot[alias[b]];
                if (need_pw[b]) pw_slot[b] = pw_slot[alias[b]];
                check((!need_up[b] || up_slot[b] >= 0) && (!need_pw[b] || pw_slot[b] >= 0), "translate storage");
            }
            for (int b : P.level_boxes[l])
                if (incoming[b] || leaf_eval[b]) down_slot[b] = n_down_++;
        }
    }

    phase("tables");
    // ------------------------------------------------------------------ tables
    {
        std::vector<double> c2p((size_t)8 * 3 * p * p);
        for (int c = 0; c < 8; ++c)
            for (int d = 0; d < 3; ++d)
                for (int a = 0; a < p; ++a)
                    for (int i = 0; i < p; ++i)
                        c2p[((size_t)c * 3 + d) * p * p + a + (size_t)p * i] = P.p2c[((size_t)c * 3 + d) * p * p + i + (size_t)p * a];
        c2p_ = upload(c2p);
        p2c_ = upload(P.p2c);
        lev_.resize(P.nlevels);
        for (int l = 0; l < P.nlevels; ++l) {
            const auto& T = P.lev[l];
            std::vector<cd> a((size_t)n * p), h((size_t)n2 * p), bt((size_t)p * n), btw((size_t)p * n2);
            for (int k = 0; k < n; ++k)
                for (int m = 0; m < p; ++m) {
                    const cplx v = T.poly2pw[k + (size_t)n * m];
                    a[k + (size_t)n * m] = cd{v.real(), v.imag()};
                    if (k < n2) h[k + (size_t)n2 * m] = cd{v.real(), v.imag()};
                    const cplx u = T.pw2poly[k + (size_t)n * m];
                    bt[m + (size_t)p * k] = cd{u.real(), u.imag()};
                    if (k < n2) {
                        const double w = k >= n / 2 ? 0.5 : 1.0;
                        btw[m + (size_t)p * k] = cd{w * u.real(), w * u.imag()};
                    }
                }
            lev_[l].poly2pw = upload(a);
            lev_[l].poly2pw_half = upload(h);
            lev_[l].pw2polyT = upload(bt);
            lev_[l].pw2polyTw = upload(btw);
            lev_[l].shift = upload(T.shift);
        }
    }

    phase("upward: proxy moment");
    // ------------------------------------------------------------------ upward: proxy moments
    {
        std::vector<std::vector<int>> by_center(P.nboxes);
        for (int w = 0; w < (int)P.c2proxy_work.size(); ++w) by_center[P.c2proxy_work[w].center_box].push_back(w);
        std::vector<int> slot, rng{0}, s0, sc;
        std::vector<double4> cs;
        for (int b = 0; b < P.nboxes; ++b) {
            if (by_center[b].empty() || up_slot[b] < 0 || alias[b] >= 0) continue;
            slot.push_back((int)up_slot[b]);
            const int lvl = P.c2proxy_work[by_center[b][0]].level;
            cs.push_back(make_double4(P.centers[3 * b], P.centers[3 * b + 1], P.centers[3 * b + 2], 2.0 / P.boxsize[lvl]));
            for (int w : by_center[b]) {
                const auto& W2 = P.c2proxy_work[w];
                check(W2.level == lvl, "work level");
                check(P.src_start[W2.src_box] >= 0 && P.src_start[W2.src_box] + P.src_count[W2.src_box] <= n_all_,
                      "work source range");
                s0.push_back(P.src_start[W2.src_box]);
                sc.push_back(P.src_count[W2.src_box]);
            }
            rng.push_back((int)s0.size());
        }
        c2x_.src = src_;
        c2x_.proxy_up = proxy_up_;
        c2x_.n_centers = (int)slot.size();
        c2x_.slot = upload(slot);
        c2x_.center_scale = upload(cs);
        c2x_.rng_start = upload(rng);
        c2x_.src_start = upload(s0);
        c2x_.src_count = upload(sc);
        launches_ += 1;
    }
    phase("upward: c2p groups");
    // ------------------------------------------------------------------ upward: c2p groups
    for (int l = P.nlevels - 1; l >= 0; --l) {
        for (int c = 0; c < 8; ++c) {
            std::vector<int64_t> in, out;
            for (int b : P.level_boxes[l]) {
                if (!P.has_proxy_from_children[b] || up_slot[b] < 0 || alias[b] >= 0) continue;
                const int ch = P.children[b][c];
                if (ch < 0 || !(P.src_count[ch] > 0 && P.ifpwexp[ch])) continue;
                check(up_slot[ch] >= 0, "c2p offsets");
                in.push_back(up_slot[ch] * ncoef);
                out.push_back(up_slot[b] * ncoef);
            }
            if (in.empty()) continue;
            C2PGroup g;
            g.n = (int)in.size();
            g.in_off = upload(in);
            g.out_off = upload(out);
            g.child = c;
            c2p_groups_.push_back(g);
        }
    }
    phase("outgoing plane waves");
    // ------------------------------------------------------------------ outgoing plane waves
    for (int l = 0; l < P.nlevels; ++l) {
        std::vector<int64_t> in, out;
        for (int b : P.level_boxes[l]) {
            if (pw_slot[b] < 0 || alias[b] >= 0) continue;
            check(up_slot[b] >= 0, "pw box without proxy");
            in.push_back(up_slot[b] * ncoef);
            out.push_back(pw_slot[b] * M);
        }
        if (in.empty()) continue;
        PwGroup g;
        g.level = l;
        g.n = (int)in.size();
        g.in_off = upload(in);
        g.out_off = upload(out);
        pw_groups_.push_back(g);
    }
    phase("downward per level");
    // ------------------------------------------------------------------ downward per level
    for (int l = 0; l < P.nlevels; ++l) {
        const double bs = P.boxsize[l];
        std::vector<int> ts{0}, tslot, tst;
        std::vector<int64_t> down, pin, pout, pmat;
        for (int b : P.level_boxes[l]) {
            if (!incoming[b]) continue;
            tslot.push_back((int)pw_slot[b]);
            tst.push_back(13);
            for (int ind = 0; ind < 27; ++ind) {
                const int nb = P.colleagues[b][ind];
                if (nb < 0 || nb == b) continue;
                if (P.is_leaf[b] && P.is_leaf[nb]) continue;
                if (P.pw_off[nb] < 0) continue;
                int st = 0, stride = 1;
                for (int d = 0; d < 3; ++d) {
                    const int kd = (int)std::lround((P.centers[3 * b + d] - P.centers[3 * nb + d]) / bs) + 1;
                    check(kd >= 0 && kd <= 2, "shift stencil");
                    st += kd * stride;
                    stride *= 3;
                }
                check(pw_slot[nb] >= 0, "colleague plane waves");
                tslot.push_back((int)pw_slot[nb]);
                tst.push_back(st);
            }
            ts.push_back((int)tslot.size());
            down.push_back(down_slot[b] * ncoef);
            if (!P.iftensprodeval[b]) {
                for (int c = 0; c < 8; ++c) {
                    const int ch = P.children[b][c];
                    // children that neither receive incoming expansions nor evaluate read nothing
                    if (ch < 0 || !(P.src_count[ch] + P.trg_count[ch]) || down_slot[ch] < 0) continue;
                    pin.push_back(down_slot[b] * ncoef);
                    pout.push_back(down_slot[ch] * ncoef);
                    pmat.push_back((int64_t)c * 3 * p * p);
                }
            }
        }
        if (down.empty()) continue;
        EvalLevel E;
        E.level = l;
        E.n = (int)down.size();
        E.term_start = upload(ts);
        E.term_slot = upload(tslot);
        E.term_stencil = upload(tst);
        E.down_off = upload(down);
        E.n_p2c = (int)pin.size();
        if (E.n_p2c) {
            E.p2c_in = upload(pin);
            E.p2c_out = upload(pout);
            E.p2c_mat = upload(pmat);
        }
        eval_levels_.push_back(E);
    }
    phase("leaf evaluation");
    // ------------------------------------------------------------------ leaf evaluation
    {
        std::vector<int> slot, t0, tc;
        std::vector<double4> cs;
        for (int b = 0; b < P.nboxes; ++b) {
            if (!leaf_eval[b]) continue;
            slot.push_back((int)down_slot[b]);
            t0.push_back(P.trg_start[b]);
            tc.push_back(P.trg_count[b]);
            cs.push_back(make_double4(P.centers[3 * b], P.centers[3 * b + 1], P.centers[3 * b + 2], 2.0 / P.boxsize[P.depth[b]]));
        }
        eval_.trg = trg_;
        eval_.proxy_down = nullptr;  // the multi-RHS path passes its own coefficients
        eval_.pot = pot_sorted_;
        eval_.n_leaves = (int)slot.size();
        for (int c : tc) eval_max_trg_ = std::max(eval_max_trg_, c);
        eval_.slot = upload(slot);
        eval_.trg_start = upload(t0);
        eval_.trg_count = upload(tc);
        eval_leaf_trg_ = tc;
        eval_.center_scale = upload(cs);
    }
    phase("FP64 single-RHS pass");
    // ------------------------------------------------------------------ FP64 single-RHS pass by level
    // Same boxes and translations as the lists above, renumbered so that each
    // level's plane waves and downward coefficients live in level-sized
    // buffers.  The reference runs the downward pass in the same level order
    // (form_eval_expansions per level, cpp/src/dmk/pbc_tree.cpp:1705-1709; its
    // body, :1253-1430, shifts, converts to proxy coefficients, translates to
    // the children and evaluates the leaves of one level).
    {
        std::vector<int64_t> loc_down(P.nboxes, -1), loc_pw(P.nboxes, -1);
        f64_levels_.resize(P.nlevels);
        for (int l = 0; l < P.nlevels; ++l) {
            int64_t nd = 0, np = 0;
            for (int b : P.level_boxes[l]) {
                check(P.depth[b] == l, "level box depth");
                if (down_slot[b] >= 0) loc_down[b] = nd++;
                if (pw_slot[b] >= 0 && alias[b] < 0) loc_pw[b] = np++;
            }
            for (int b : P.level_boxes[l])
                if (pw_slot[b] >= 0 && alias[b] >= 0) loc_pw[b] = loc_pw[alias[b]];
            f64_levels_[l].level = l;
            f64_levels_[l].n_down = nd;
            down_level_boxes_[l & 1] = std::max(down_level_boxes_[l & 1], nd);
            pw_level_boxes_ = std::max(pw_level_boxes_, np);
        }
        for (int l = 0; l < P.nlevels; ++l) {
            Fp64Level& F = f64_levels_[l];
            const double bs = P.boxsize[l];
            std::vector<int64_t> pin, pout;
            for (int b : P.level_boxes[l]) {
                if (pw_slot[b] < 0 || alias[b] >= 0) continue;
                pin.push_back(up_slot[b] * ncoef);
                pout.push_back(loc_pw[b] * M);
            }
            F.n_pw = (int)pin.size();
            if (F.n_pw) {
                F.pw_in_off = upload(pin);
                F.pw_out_off = upload(pout);
            }
            std::vector<int> ts{0}, tslot, tst;
            std::vector<int64_t> down, cin, cout, cmat;
            std::vector<int> slot, t0, tc;
            std::vector<double4> cs;
            for (int b : P.level_boxes[l]) {
                if (leaf_eval[b]) {
                    slot.push_back((int)loc_down[b]);
                    t0.push_back(P.trg_start[b]);
                    tc.push_back(P.trg_count[b]);
                    cs.push_back(make_double4(P.centers[3 * b], P.centers[3 * b + 1], P.centers[3 * b + 2], 2.0 / bs));
                }
                if (!incoming[b]) continue;
                tslot.push_back((int)loc_pw[b]);
                tst.push_back(13);
                for (int ind = 0; ind < 27; ++ind) {
                    const int nb = P.colleagues[b][ind];
                    if (nb < 0 || nb == b) continue;
                    if (P.is_leaf[b] && P.is_leaf[nb]) continue;
                    if (P.pw_off[nb] < 0) continue;
                    check(P.depth[nb] == l && loc_pw[nb] >= 0, "colleague plane waves");
                    int st = 0, stride = 1;
                    for (int d = 0; d < 3; ++d) {
                        const int kd = (int)std::lround((P.centers[3 * b + d] - P.centers[3 * nb + d]) / bs) + 1;
                        check(kd >= 0 && kd <= 2, "shift stencil");
                        st += kd * stride;
                        stride *= 3;
                    }
                    tslot.push_back((int)loc_pw[nb]);
                    tst.push_back(st);
                }
                ts.push_back((int)tslot.size());
                down.push_back(loc_down[b] * ncoef);
                if (!P.iftensprodeval[b]) {
                    for (int c = 0; c < 8; ++c) {
                        const int ch = P.children[b][c];
                        if (ch < 0 || !(P.src_count[ch] + P.trg_count[ch]) || loc_down[ch] < 0) continue;
                        check(P.depth[ch] == l + 1 && l + 1 < P.nlevels, "p2c child level");
                        cin.push_back(loc_down[b] * ncoef);
                        cout.push_back(loc_down[ch] * ncoef);
                        cmat.push_back((int64_t)c * 3 * p * p);
                    }
                }
            }
            F.n_in = (int)down.size();
            if (F.n_in) {
                F.term_start = upload(ts);
                F.term_slot = upload(tslot);
                F.term_stencil = upload(tst);
                F.down_off = upload(down);
            }
            F.n_p2c = (int)cin.size();
            if (F.n_p2c) {
                F.p2c_in = upload(cin);
                F.p2c_out = upload(cout);
                F.p2c_mat = upload(cmat);
            }
            F.eval.trg = trg_;
            F.eval.pot = pot_sorted_;
            F.eval.n_leaves = (int)slot.size();
            if (F.eval.n_leaves) {
                F.eval.slot = upload(slot);
                F.eval.trg_start = upload(t0);
                F.eval.trg_count = upload(tc);
                F.eval.center_scale = upload(cs);
            }
        }
        int64_t leaves = 0;
        for (const auto& F : f64_levels_) leaves += F.eval.n_leaves;
        check(leaves == eval_.n_leaves, "leaf evaluation lists by level");
    }
    phase("near field");
    // ------------------------------------------------------------------ near field
    {
        // Contact-geometry cull of the reference (cpp/include/dmk/tree.hpp:111-220,
        // applied at cpp/src/dmk/pbc_tree.cpp:1528-1563), used here only to count
        // the pairs the reference evaluates: a point is kept if its squared
        // distance to the shared face/edge/corner of the two boxes is < b^2.
        int filter_min = 64;
        if (const char* fs = std::getenv("DMK_FILTER_NTRG_MIN")) filter_min = std::atoi(fs);
        auto count_in_range = [&](int sb, int tb, double d2max, bool sources) {
            const double sa = P.boxsize[P.depth[sb]], sbb = P.boxsize[P.depth[tb]];
            int tdim[3], nt = 0, odim[3], no = 0;
            double tco[3], olo[3], ohi[3];
            for (int d = 0; d < 3; ++d) {
                const double a = P.centers[3 * sb + d] - sa / 2, b = P.centers[3 * tb + d] - sbb / 2;
                if (a + sa == b) {
                    tdim[nt] = d; tco[nt++] = b;
                } else if (b + sbb == a) {
                    tdim[nt] = d; tco[nt++] = a;
                } else {
                    odim[no] = d; olo[no] = std::max(a, b); ohi[no++] = std::min(a + sa, b + sbb);
                }
            }
            const double* pts = sources ? P.src_sorted.data() : P.trg_sorted.data();
            const int s0 = sources ? P.src_start[sb] : P.trg_start[tb];
            const int cnt = sources ? P.src_count[sb] : P.trg_count[tb];
            int64_t kept = 0;
            for (int i = s0; i < s0 + cnt; ++i) {
                const double* x = pts + 3 * (size_t)i;
                double d2 = 0;
                for (int k = 0; k < nt; ++k) d2 += (x[tdim[k]] - tco[k]) * (x[tdim[k]] - tco[k]);
                for (int k = 0; k < no; ++k) {
                    const double c = std::min(std::max(x[odim[k]], olo[k]), ohi[k]);
                    d2 += (x[odim[k]] - c) * (x[odim[k]] - c);
                }
                if (d2 < d2max) kept++;
            }
            return kept;
        };
        std::vector<int> t0, tc, ps{0}, s0, sc, pcb;
        std::vector<double> bsz;
        // float bounding boxes (rounded outwards) of every 32-source chunk of the
        // source boxes that appear in near pairs, one entry set per box
        std::vector<int> box_cb(P.nboxes, -1);
        std::vector<float4> clo, chi;
        auto chunk_base = [&](int sb) {
            if (box_cb[sb] >= 0) return box_cb[sb];
            box_cb[sb] = (int)clo.size();
            const int st = P.src_start[sb], cnt = P.src_count[sb];
            for (int j0 = 0; j0 < cnt; j0 += dev::kNearTcChunk) {
                double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
                for (int i = st + j0; i < st + std::min(cnt, j0 + dev::kNearTcChunk); ++i)
                    for (int d = 0; d < 3; ++d) {
                        lo[d] = std::min(lo[d], P.src_sorted[3 * (size_t)i + d]);
                        hi[d] = std::max(hi[d], P.src_sorted[3 * (size_t)i + d]);
                    }
                float l[3], h[3];
                for (int d = 0; d < 3; ++d) {
                    l[d] = std::nextafter((float)lo[d], -INFINITY);
                    h[d] = std::nextafter((float)hi[d], INFINITY);
                }
                clo.push_back(make_float4(l[0], l[1], l[2], 0.0f));
                chi.push_back(make_float4(h[0], h[1], h[2], 0.0f));
            }
            return box_cb[sb];
        };
        for (int tb : P.direct_work) {
            if (P.trg_count[tb] == 0) continue;
            t0.push_back(P.trg_start[tb]);
            tc.push_back(P.trg_count[tb]);
            const int tl = P.depth[tb];
            for (int li = P.list1_start[tb]; li < P.list1_start[tb + 1]; ++li) {
                const int sb = P.list1[li];
                const int sl = P.depth[sb];
                double b = P.boxsize[sl];
                if (P.ifpwexp[sb] && sb == tb)
                    b /= 2.0;
                else if (sl < tl)
                    b = P.boxsize[tl];
                check(P.src_start[sb] >= 0 && P.src_start[sb] + P.src_count[sb] <= n_all_, "near source range");
                {
                    const bool src_larger = sl < tl, trg_larger = sl > tl;
                    const bool filter_same = !src_larger && !trg_larger && filter_min >= 0 && P.trg_count[tb] >= filter_min;
                    const int64_t ns = (src_larger || filter_same) ? count_in_range(sb, tb, b * b, true) : P.src_count[sb];
                    const int64_t ntg = trg_larger ? count_in_range(sb, tb, b * b, false) : P.trg_count[tb];
                    near_pairs_culled_ += ns * ntg;
                    near_pairs_nominal_ += (int64_t)P.src_count[sb] * P.trg_count[tb];
                }
                s0.push_back(P.src_start[sb]);
                sc.push_back(P.src_count[sb]);
                bsz.push_back(b);
                pcb.push_back(P.src_count[sb] > 0 ? chunk_base(sb) : 0);
            }
            ps.push_back((int)s0.size());
        }
        near_leaf_cost_.assign(tc.size(), 0);
        int64_t near_targets = 0;
        for (size_t i = 0; i < tc.size(); ++i) {
            int64_t ns = 0;
            for (int k = ps[i]; k < ps[i + 1]; ++k) ns += sc[k];
            near_leaf_cost_[i] = (int64_t)tc[i] * ns;
            near_targets += tc[i];
        }
        check(near_targets == n_, "near-field leaves cover every target once");
        for (size_t i = 0; i < tc.size(); ++i) {
            near_max_trg_ = std::max(near_max_trg_, tc[i]);
            near_max_pairs_ = std::max(near_max_pairs_, ps[i + 1] - ps[i]);
            int ch = 0;
            for (int k = ps[i]; k < ps[i + 1]; ++k) ch += (sc[k] + dev::kNearTcChunk - 1) / dev::kNearTcChunk;
            near_max_chunks_ = std::max(near_max_chunks_, ch);
        }
        near_pair_chunk_base_ = upload(pcb);
        near_chunk_lo_ = upload(clo);
        near_chunk_hi_ = upload(chi);
        near_.pair_chunk_base = near_pair_chunk_base_;
        near_.chunk_lo = near_chunk_lo_;
        near_.chunk_hi = near_chunk_hi_;
        near_.trg = trg_;
        near_.src = src_;
        near_.pot = pot_sorted_;
        near_.n_leaves = (int)t0.size();
        near_.trg_start = upload(t0);
        near_.trg_count = upload(tc);
        near_.pair_start = upload(ps);
        near_.pair_src_start = upload(s0);
        near_.pair_src_count = upload(sc);
        near_.pair_bsize = upload(bsz);
        check(P.resid.size() <= 32, "residual polynomial length");
        near_.nc = (int)P.resid.size();
        for (int i = 0; i < near_.nc; ++i) near_.coef[i] = P.resid[i];
        launches_ += 1;
    }

    phase("FP64 transform scrat");
    // ------------------------------------------------------------------ FP64 transform scratch
    // Enough for the largest level in one chunk, capped at PDMK_FP64_SCRATCH_MB
    // (default 1024 MiB); larger levels run in chunks of boxes.
    {
        int64_t budget_mb = 1024;
        if (const char* e = std::getenv("PDMK_FP64_SCRATCH_MB")) budget_mb = std::max<int64_t>(16, std::atoll(e));
        const int64_t budget = (budget_mb << 20) / (int64_t)sizeof(cd);
        int64_t want = 1;
        for (const auto& F : f64_levels_) {
            want = std::max(want, fp64_need_pw_out() * F.n_pw);
            want = std::max(want, fp64_need_pw_in() * F.n_in);
            want = std::max(want, fp64_need_c2p() * F.n_p2c);
        }
        for (const auto& g : c2p_groups_) want = std::max(want, fp64_need_c2p() * g.n);
        f64_scratch_elems_ = std::min(want, std::max(budget, fp64_need_max()));
        const Fp64Chunks C = fp64_chunks(f64_scratch_elems_);
        const bool fc = dev::sep3_supported<double>(p), fpw = dev::pw_fused_supported<double>(p, n, n2);
        auto nchunks = [](int64_t nb, int c) { return (int)((nb + c - 1) / c); };
        for (const auto& g : c2p_groups_) launches_ += fc ? 1 : 3 * nchunks(g.n, C.c2p);
        for (const auto& F : f64_levels_) {
            if (F.n_pw) launches_ += fpw ? 1 : 3 * nchunks(F.n_pw, C.pw_out);
            if (F.n_in) launches_ += (fpw ? 2 : 4) * nchunks(F.n_in, C.pw_in);
            if (F.n_p2c) launches_ += fc ? 1 : 3 * nchunks(F.n_p2c, C.c2p);
            if (F.eval.n_leaves) launches_ += 1;
        }
    }
    if (fp64_working_set && !P.qp) {  // quasi-periodic trees evaluate on the two-column state
        ensure_fp64_working_set();
        noalloc_reserve(device_);  // double trees may use the no-allocation evaluate
    }

    phase("far field");
    // ------------------------------------------------------------------ far field
    {
        n_grid_ = (int64_t)ng[0] * ng[1] * ng[2];
        n_spec_ = (int64_t)ng[0] * ng[1] * (ng[2] / 2 + 1);
        grid_ = alloc<double>(n_grid_);
        spec_ = alloc<cd>(n_spec_);
        // multiplier: 1/2 (in K(k) + in K(-k)) w(k) H^2 / Psi(k)^2
        const double es_beta = 2.30 * W;
        std::vector<double> gx(200), gw(200);
        gauss_legendre(200, gx.data(), gw.data());
        auto phihat = [&](int d, int k) {
            const double h = 2.0 * M_PI / ng[d], alpha = 0.5 * W * h;
            double s = 0;
            for (int i = 0; i < 200; ++i) {
                const double z = gx[i];
                s += gw[i] * std::exp(es_beta * (std::sqrt(1.0 - z * z) - 1.0)) * std::cos(k * alpha * z);
            }
            return alpha * s;
        };
        std::vector<double> ph[3];
        for (int d = 0; d < 3; ++d) {
            ph[d].resize(ng[d]);
            for (int i = 0; i < ng[d]; ++i) ph[d][i] = phihat(d, i <= ng[d] / 2 ? i : i - ng[d]);
        }
        const double H = std::pow(2.0 * M_PI, 3) / ((double)ng[0] * ng[1] * ng[2]);
        const double* u = P.umat;
        const double a11 = 1.0 / u[0], a21 = -u[3] / (u[0] * u[4]), a22 = 1.0 / u[4];
        const double a31 = (u[3] * u[7] - u[6] * u[4]) / (u[0] * u[4] * u[8]);
        const double a32 = -u[7] / (u[4] * u[8]), a33 = 1.0 / u[8];
        const Pswf0& pf = Pswf0::get(P.dp.beta);
        const double psi0 = pf(0.0), twopi = 2.0 * M_PI;
        const double dfac = 4.0 * M_PI / (psi0 * P.volume);
        auto inK = [&](int k1, int k2, int k3) {
            return k1 >= -P.ms / 2 && k1 <= (P.ms - 1) / 2 && k2 >= -P.mt / 2 && k2 <= (P.mt - 1) / 2 && k3 >= -P.mu / 2 &&
                   k3 <= (P.mu - 1) / 2;
        };
        std::vector<double> mult(n_spec_, 0.0);
        const int n3h = ng[2] / 2 + 1;
        for (int i1 = 0; i1 < ng[0]; ++i1)
            for (int i2 = 0; i2 < ng[1]; ++i2)
                for (int i3 = 0; i3 < n3h; ++i3) {
                    const int k1 = i1 <= ng[0] / 2 ? i1 : i1 - ng[0];
                    const int k2 = i2 <= ng[1] / 2 ? i2 : i2 - ng[1];
                    const int k3 = i3;
                    const double frac = 0.5 * ((inK(k1, k2, k3) ? 1 : 0) + (inK(-k1, -k2, -k3) ? 1 : 0));
                    if (frac == 0) continue;
                    const double d1 = twopi * (a11 * k1);
                    const double d2 = twopi * (a21 * k1 + a22 * k2);
                    const double d3 = twopi * (a31 * k1 + a32 * k2 + a33 * k3);
                    const double kk = d1 * d1 + d2 * d2 + d3 * d3;
                    if (kk < 1e-30) continue;
                    const double xval = std::sqrt(kk) * P.rc / P.dp.beta;
                    if (xval > 1.0) continue;
                    const double w = dfac * pf(xval) / kk;
                    const double Ps = ph[0][i1] * ph[1][i2] * ph[2][i3];
                    mult[((size_t)i1 * ng[1] + i2) * n3h + i3] = frac * w * H * H / (Ps * Ps);
                }
        mult_ = upload(mult);
        if (P.qp) {
            // Quasi-periodic multiplier (cpp/src/dmk/pbc.cpp:289-318): the
            // spectrum of the phased charges is weighted by w(2 pi L^-T k + bloch)
            // over the mode box, which is not even in k.  Over the stored half
            // spectrum of the two real transforms (real and imaginary part of
            // the phased charges) it enters through its even and odd parts
            // s = (w(k) + w(-k)) / 2 and d = (w(k) - w(-k)) / 2.
            auto wq = [&](int k1, int k2, int k3) {
                if (!inK(k1, k2, k3)) return 0.0;
                const double d1 = twopi * (a11 * k1) + P.bloch[0];
                const double d2 = twopi * (a21 * k1 + a22 * k2) + P.bloch[1];
                const double d3 = twopi * (a31 * k1 + a32 * k2 + a33 * k3) + P.bloch[2];
                const double kk = d1 * d1 + d2 * d2 + d3 * d3;
                if (kk < 1e-30) return 0.0;
                const double xval = std::sqrt(kk) * P.rc / P.dp.beta;
                return xval > 1.0 ? 0.0 : dfac * pf(xval) / kk;
            };
            std::vector<double> qs(n_spec_, 0.0), qd(n_spec_, 0.0);
            for (int i1 = 0; i1 < ng[0]; ++i1)
                for (int i2 = 0; i2 < ng[1]; ++i2)
                    for (int i3 = 0; i3 < n3h; ++i3) {
                        const int k1 = i1 <= ng[0] / 2 ? i1 : i1 - ng[0];
                        const int k2 = i2 <= ng[1] / 2 ? i2 : i2 - ng[1];
                        const int k3 = i3;
                        const double wp = wq(k1, k2, k3), wm = wq(-k1, -k2, -k3);
                        if (wp == 0.0 && wm == 0.0) continue;
                        const double Ps = ph[0][i1] * ph[1][i2] * ph[2][i3];
                        const double c = H * H / (Ps * Ps);
                        const size_t at = ((size_t)i1 * ng[1] + i2) * n3h + i3;
                        qs[at] = 0.5 * (wp + wm) * c;
                        qd[at] = 0.5 * (wp - wm) * c;
                    }
            qp_s_ = upload(qs);
            qp_d_ = upload(qd);
            // Bloch phases: e^{i bloch.R} of each sorted source (R = its lattice
            // image vector) and e^{i bloch.x} of each sorted target
            std::vector<double2> sp(n_all_), tp(n_);
            for (int j = 0; j < n_all_; ++j) {
                const int q = P.src_charge_idx[j];
                double ph_j = 0.0;
                for (int d = 0; d < 3; ++d)
                    ph_j += P.bloch[d] * (P.src_sorted[3 * (size_t)j + d] - P.r_user[3 * (size_t)q + d]);
                sp[j] = make_double2(std::cos(ph_j), std::sin(ph_j));
            }
            for (int t = 0; t < n_; ++t) {
                const int u = P.trg_perm[t];
                double th = 0.0;
                for (int d = 0; d < 3; ++d) th += P.bloch[d] * P.r_user[3 * (size_t)u + d];
                tp[t] = make_double2(std::cos(th), std::sin(th));
            }
            qp_src_phase_ = upload(sp);
            qp_trg_phase_ = upload(tp);
            qp_ = true;
        }
        for (int i = 0; i < 9; ++i) {
            frame_.qmat[i] = P.qmat[i];
            frame_.umatinv[i] = P.umatinv[i];
        }
        CUFFT_CHECK(cufftPlan3d(&plan_fwd_, ng[0], ng[1], ng[2], CUFFT_D2Z));
        CUFFT_CHECK(cufftPlan3d(&plan_inv_, ng[0], ng[1], ng[2], CUFFT_Z2D));
        CUFFT_CHECK(cufftSetStream(plan_fwd_, stream_));
        CUFFT_CHECK(cufftSetStream(plan_inv_, stream_));

        std::vector<int> bs, bc;
        std::vector<int4> bo, be;
        for (auto& bn : bins) {
            bs.push_back(bn.start);
            bc.push_back(bn.count);
            bo.push_back(bn.org);
            be.push_back(bn.ext);
            nufft_max_jk_ = std::max(nufft_max_jk_, bn.ext.y * bn.ext.z);
            nufft_max_ex_ = std::max(nufft_max_ex_, bn.ext.x);
            nufft_max_cells_ = std::max(nufft_max_cells_, bn.ext.x * bn.ext.y * bn.ext.z);
        }
        nufft_.n_leaves = (int)bins.size();
        nufft_.max_cells = nufft_max_cells_;
        nufft_.trg_start = upload(bs);
        nufft_.trg_count = upload(bc);
        nufft_.sub_origin = upload(bo);
        nufft_.sub_extent = upload(be);
        nufft_.pt_t = upload(pt_t);
        nufft_.pt_l0 = upload(pt_l0);
        {
            // interpolation order: inside each bin, targets by window cell
            // (x, y, z), stable; the tree keeps its own target order
            std::vector<int> order(n_);
            std::iota(order.begin(), order.end(), 0);
            for (auto& bn : bins) {
                auto key = [&](int t) {
                    const int4 l = pt_l0[t];
                    return (((int64_t)(l.x - bn.org.x) << 20) | ((int64_t)(l.y - bn.org.y) << 10)) + (l.z - bn.org.z);
                };
                std::stable_sort(order.begin() + bn.start, order.begin() + bn.start + bn.count,
                                 [&](int x, int y) { return key(x) < key(y); });
            }
            nufft_.interp_order = upload(order);
            std::vector<int2> ipair;
            std::vector<int> bin_pair{0};
            for (auto& bn : bins) {
                for (int i = bn.start; i < bn.start + bn.count;) {
                    const int ta = order[i];
                    int tb = -1;
                    if (i + 1 < bn.start + bn.count) {
                        const int4 la = pt_l0[ta], lb = pt_l0[order[i + 1]];
                        if (la.x == lb.x && la.y == lb.y && la.z == lb.z) tb = order[i + 1];
                    }
                    ipair.push_back(make_int2(ta, tb));
                    i += tb >= 0 ? 2 : 1;
                }
                bin_pair.push_back((int)ipair.size());
                nufft_.max_pairs = std::max(nufft_.max_pairs, bin_pair.back() - bin_pair[bin_pair.size() - 2]);
            }
            if (ipair.empty()) ipair.push_back(make_int2(0, -1));
            nufft_.interp_pair = upload(ipair);
            nufft_.bin_pair = upload(bin_pair);
            // spreading runs: inside each bin, targets by (y, z, x) window start;
            // a run = equal (y, z), x offsets within kSpreadRunDx of its first
            std::vector<int> sorder(n_);
            std::iota(sorder.begin(), sorder.end(), 0);
            std::vector<int4> runs;
            std::vector<int> bin_run{0};
            for (auto& bn : bins) {
                auto key = [&](int t) {
                    const int4 l = pt_l0[t];
                    return (((int64_t)(l.y - bn.org.y) << 20) | ((int64_t)(l.z - bn.org.z) << 10)) + (l.x - bn.org.x);
                };
                std::stable_sort(sorder.begin() + bn.start, sorder.begin() + bn.start + bn.count,
                                 [&](int x, int y) { return key(x) < key(y); });
                for (int i = bn.start; i < bn.start + bn.count;) {
                    const int4 l = pt_l0[sorder[i]];
                    int j = i;
                    while (j < bn.start + bn.count) {
                        const int4 m = pt_l0[sorder[j]];
                        if (m.y != l.y || m.z != l.z || m.x - l.x > dev::kSpreadRunDx) break;
                        ++j;
                    }
                    check(l.y - bn.org.y >= 0 && l.y - bn.org.y < 0x8000 && l.z - bn.org.z >= 0 &&
                              l.z - bn.org.z < 0x8000 && l.x >= bn.org.x,
                          "spreading run offsets");
                    runs.push_back(make_int4(i, j - i, (l.y - bn.org.y) | ((l.z - bn.org.z) << 16), l.x - bn.org.x));
                    i = j;
                }
                bin_run.push_back((int)runs.size());
            }
            if (runs.empty()) runs.push_back(make_int4(0, 0, 0, 0));
            nufft_.spread_order = upload(sorder);
            nufft_.spread_run = upload(runs);
            nufft_.bin_run = upload(bin_run);
        }
        nufft_.q_sorted = q_sorted_;
        nufft_.grid = grid_;
        nufft_.far = far_sorted_;
        nufft_.n1 = ng[0];
        nufft_.n2 = ng[1];
        nufft_.n3 = ng[2];
        nufft_.w = W;
        nufft_.es_beta = es_beta;
        launches_ += 4;  // gather_q, spread, multiply, interp (the two cuFFT transforms are library kernels)
    }
    launches_ += 2;  // charge gather, final gather
    PDMK_CUDA_CHECK(cudaStreamSynchronize(stream_));
    phase("");
}

DeviceTree::~DeviceTree() { release(); }

void DeviceTree::ensure_fp64_working_set() {
    if (proxy_up_) return;
    const int64_t ncoef = (int64_t)p_ * p_ * p_;
    proxy_up_ = alloc<double>(n_up_ * ncoef);
    down_level_[0] = alloc<double>(std::max<int64_t>(down_level_boxes_[0], 1) * ncoef);
    down_level_[1] = alloc<double>(std::max<int64_t>(down_level_boxes_[1], 1) * ncoef);
    pw_level_ = alloc<cd>(std::max<int64_t>(pw_level_boxes_, 1) * (int64_t)M_);
    f64_scratch_ = alloc<cd>(f64_scratch_elems_);
    c2x_.proxy_up = proxy_up_;
}

int64_t DeviceTree::fp64_need_c2p() const {
    const int64_t ncoef = (int64_t)p_ * p_ * p_;
    return dev::sep3_supported<double>(p_) ? 0 : 2 * ((ncoef + 1) / 2);
}
int64_t DeviceTree::fp64_need_pw_out() const {
    const int64_t p = p_, n = npw_;
    return dev::pw_fused_supported<double>(p_, npw_, npw2_) ? 0 : p * p * n + p * n * n;
}
int64_t DeviceTree::fp64_need_pw_in() const {
    const int64_t p = p_, n = npw_, n2 = npw2_;
    return (int64_t)M_ + (dev::pw_fused_supported<double>(p_, npw_, npw2_) ? 0 : n * n2 * p + n2 * p * p);
}
int64_t DeviceTree::fp64_need_max() const {
    return std::max({fp64_need_c2p(), fp64_need_pw_out(), fp64_need_pw_in()});
}

DeviceTree::Fp64Chunks DeviceTree::fp64_chunks(int64_t cap) const {
    auto c = [cap](int64_t need) {
        if (need <= 0) return (int)INT32_MAX;
        return (int)std::min<int64_t>(INT32_MAX, std::max<int64_t>(1, cap / need));
    };
    Fp64Chunks r;
    r.c2p = c(fp64_need_c2p());
    r.pw_out = c(fp64_need_pw_out());
    r.pw_in = c(fp64_need_pw_in());
    return r;
}

int DeviceTree::run_fp64_tree(const double* q, cd* scratch, int64_t cap, cudaStream_t s) {
    const int p = p_, n = npw_, n2 = npw2_, M = M_;
    const int64_t ncoef = (int64_t)p * p * p;
    const int64_t ncoef_c = (ncoef + 1) / 2;  // a real (p,p,p) tensor in complex-sized slots
    const bool fused_c2p = dev::sep3_supported<double>(p);
    const bool fused_pw = dev::pw_fused_supported<double>(p, n, n2);
    const Fp64Chunks C = fp64_chunks(cap);
    int nl = 0;
    PDMK_CUDA_CHECK(cudaMemsetAsync(proxy_up_, 0, sizeof(double) * std::max<int64_t>(n_up_ * ncoef, 1), s));
    dev::launch_gather(src_, src_charge_idx_, q, n_all_, s);
    if (moments_dmma_ && dev::c2proxy_dmma_supported(p))
        dev::launch_c2proxy_dmma(c2x_, p, s);
    else
        dev::launch_c2proxy(c2x_, p, s);
    nl += 2;
    // child -> parent translation of real (p,p,p) tensors: one fused kernel, or
    // three contractions through scratch in chunks of C.c2p translations
    auto translate = [&](const double* in, const int64_t* in_off, double* out, const int64_t* out_off,
                         const double* mat, const int64_t* mat_off, int count, int structure, bool accumulate) {
        if (fused_c2p) {
            dev::Sep3 f{};
            f.in = in; f.in_off = in_off; f.out = out; f.out_off = out_off; f.mat = mat; f.mat_off = mat_off;
            f.tri = structure == dev::kTriUpper ? 1 : (structure == dev::kTriLower ? 2 : 0);
            f.rhs = 1; f.accumulate = accumulate ? 1 : 0;
            dev::launch_sep3<double>(f, p, count, s);
            ++nl;
            return;
        }
        double* s1 = reinterpret_cast<double*>(scratch);
        double* s2 = reinterpret_cast<double*>(scratch + (int64_t)std::min(C.c2p, count) * ncoef_c);
        for (int c0 = 0; c0 < count; c0 += C.c2p) {
            dev::ContractArgs a{};
            a.n_entries = std::min(C.c2p, count - c0);
            // x: in (i,j,k) -> s1 (j,k,a); y: s1 -> s2 (k,a,b); z: s2 -> out (a,b,c), accumulated
            a.in = in; a.in_off = in_off + c0; a.out = s1; a.out_stride = ncoef;
            a.mat = mat; a.mat_off = mat_off ? mat_off + c0 : nullptr; a.ni = p; a.na = p; a.R = p * p;
            a.mode = dev::kStore; a.structure = structure;
            // FP64 tensor cores (DMMA) when selected, else the CUDA-core contraction
            auto rrr = [&](const dev::ContractArgs& c) {
                const bool dm = fp64_dmma_ < 0 ? p_ == 28 : fp64_dmma_ != 0;
                if (dm && dev::translate_dmma_supported(c.ni, c.na)) dev::launch_translate_dmma(c, s);
                else dev::launch_contract(c, dev::kRRR, s);
            };
            rrr(a);
            a.in = s1; a.in_off = nullptr; a.in_stride = ncoef; a.out = s2; a.mat = mat + p * p;
            rrr(a);
            a.in = s2; a.out = out; a.out_off = out_off + c0; a.mat = mat + 2 * p * p;
            a.mode = accumulate ? dev::kAdd : dev::kStore;
            rrr(a);
            nl += 3;
        }
    };
    // upward
    for (const auto& g : c2p_groups_)
        translate(proxy_up_, g.in_off, proxy_up_, g.out_off, c2p_ + (int64_t)g.child * 3 * p * p, nullptr, g.n,
                  dev::kTriUpper, true);
    // downward, one level at a time
    if (!f64_levels_.empty())
        PDMK_CUDA_CHECK(cudaMemsetAsync(down_level_[0], 0, sizeof(double) * std::max<int64_t>(f64_levels_[0].n_down * ncoef, 1), s));
    for (const auto& F : f64_levels_) {
        const auto& L = lev_[F.level];
        double* down = down_level_[F.level & 1];
        // outgoing plane waves of this level
        if (F.n_pw && fused_pw) {
            dev::PwFused f{};
            f.in = proxy_up_; f.in_off = F.pw_in_off; f.out = pw_level_; f.out_off = F.pw_out_off;
            f.mat_a = L.poly2pw; f.mat_b = L.poly2pw_half; f.rhs = 1; f.e0 = 0;
            dev::launch_pw_out_fused<double>(f, p, n, n2, F.n_pw, s);
            ++nl;
        } else if (F.n_pw) {
            cd* s1 = scratch;
            cd* s2 = scratch + (int64_t)std::min(C.pw_out, F.n_pw) * p * p * n;
            for (int c0 = 0; c0 < F.n_pw; c0 += C.pw_out) {
                dev::ContractArgs a{};
                a.n_entries = std::min(C.pw_out, F.n_pw - c0);
                a.in = proxy_up_; a.in_off = F.pw_in_off + c0; a.out = s1; a.out_stride = (int64_t)p * p * n;
                a.mat = L.poly2pw; a.ni = p; a.na = n; a.R = p * p; a.mode = dev::kStore; a.structure = dev::kParIn;
                dev::launch_contract(a, dev::kRCC, s);
                a.in = s1; a.in_off = nullptr; a.in_stride = (int64_t)p * p * n; a.out = s2;
                a.out_stride = (int64_t)p * n * n; a.R = p * n;
                dev::launch_contract(a, dev::kCCC, s);
                a.in = s2; a.in_stride = (int64_t)p * n * n; a.out = pw_level_; a.out_off = F.pw_out_off + c0;
                a.mat = L.poly2pw_half; a.na = n2; a.R = n * n;
                dev::launch_contract(a, dev::kCCC, s);
                nl += 3;
            }
        }
        // incoming: shift -> plane waves to proxy coefficients, in chunks of boxes
        if (F.n_in) {
            const int CI = C.pw_in;
            const int cmax = std::min(CI, F.n_in);
            cd* pin = scratch;
            cd* s1 = pin + (int64_t)cmax * M;
            cd* s2 = s1 + (int64_t)cmax * n * n2 * p;
            for (int c0 = 0; c0 < F.n_in; c0 += CI) {
                const int ne = std::min(CI, F.n_in - c0);
                dev::ShiftArgs sa{pw_level_, L.shift, pin, M, ne, F.term_start + c0, F.term_slot, F.term_stencil};
                dev::launch_shift(sa, s);
                ++nl;
                if (fused_pw) {
                    dev::PwFused f{};
                    f.in = pin; f.in_stride = M; f.out = down; f.out_off = F.down_off + c0;
                    f.mat_a = L.pw2polyT; f.mat_b = L.pw2polyTw; f.rhs = 1; f.e0 = 0;
                    dev::launch_pw_in_fused<double>(f, p, n, n2, ne, s);
                    ++nl;
                    continue;
                }
                dev::ContractArgs a{};
                a.n_entries = ne;
                a.in = pin; a.in_stride = M; a.out = s1; a.out_stride = (int64_t)n * n2 * p;
                a.mat = L.pw2polyT; a.ni = n; a.na = p; a.R = n * n2; a.mode = dev::kStore; a.structure = dev::kParOut;
                dev::launch_contract(a, dev::kCCC, s);
                a.in = s1; a.in_stride = (int64_t)n * n2 * p; a.out = s2; a.out_stride = (int64_t)n2 * p * p;
                a.R = n2 * p;
                dev::launch_contract(a, dev::kCCC, s);
                a.in = s2; a.in_stride = (int64_t)n2 * p * p; a.out = down; a.out_off = F.down_off + c0;
                a.mat = L.pw2polyTw; a.ni = n2; a.R = p * p; a.mode = dev::kAddRealScaled; a.scale = 2.0;
                dev::launch_contract(a, dev::kCCR, s);
                nl += 3;
            }
        }
        // leaves of this level
        if (F.eval.n_leaves) {
            dev::EvalArgs e = F.eval;
            e.proxy_down = down;
            dev::launch_eval(e, p, s);
            ++nl;
            if (grad_on_) {
                dev::launch_eval_grad(e, p, grad_sorted_, n_, s);
                ++nl;
            }
        }
        // parent -> child into the next level's buffer
        if (F.level + 1 < (int)f64_levels_.size()) {
            double* next = down_level_[(F.level + 1) & 1];
            const int64_t nd = f64_levels_[F.level + 1].n_down;
            PDMK_CUDA_CHECK(cudaMemsetAsync(next, 0, sizeof(double) * std::max<int64_t>(nd * ncoef, 1), s));
            // first write of each child's coefficients (one parent each): store
            if (F.n_p2c) translate(down, F.p2c_in, next, F.p2c_out, p2c_, F.p2c_mat, F.n_p2c, dev::kTriLower, false);
        }
    }
    return nl;
}

void DeviceTree::release() {
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    multi_[0].reset();
    multi_[1].reset();
    if (stream_) cudaStreamSynchronize(stream_);
    if (stage_q_) cudaFree(stage_q_);
    if (stage_p_) cudaFree(stage_p_);
    stage_q_ = stage_p_ = nullptr;
    stage_elems_ = 0;
    if (plan_fwd_) cufftDestroy(plan_fwd_);
    if (plan_inv_) cufftDestroy(plan_inv_);
    for (void* p : allocs_) cudaFree(p);
    for (auto& e : ev_)
        if (e) cudaEventDestroy(e);
    if (stream_) cudaStreamDestroy(stream_);
    allocs_.clear();
    plan_fwd_ = plan_inv_ = 0;
    stream_ = nullptr;
    for (auto& e : ev_) e = nullptr;
}

void DeviceTree::require_periodic(const char* what) const {
    if (qp_) throw std::logic_error(std::string(what) + ": bloch is set - use evaluate_complex()");
}

void DeviceTree::run(const double* q, double* pot) {
    require_periodic("evaluate");
    ensure_fp64_working_set();
    cudaStream_t s = stream_;
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[0], s));
    PDMK_CUDA_CHECK(cudaMemsetAsync(pot_sorted_, 0, sizeof(double) * n_, s));
    run_fp64_tree(q, f64_scratch_, f64_scratch_elems_, s);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[1], s));
    dev::launch_near(near_, s);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[2], s));
    // far field
    dev::launch_nufft_gather_q(trg_perm_, q, q_sorted_, n_, s);
    PDMK_CUDA_CHECK(cudaMemsetAsync(grid_, 0, sizeof(double) * n_grid_, s));
    dev::launch_spread(nufft_, nufft_max_jk_, nufft_max_ex_, s);
    CUFFT_CHECK(cufftExecD2Z(plan_fwd_, grid_, reinterpret_cast<cufftDoubleComplex*>(spec_)));
    dev::launch_multiply(spec_, mult_, n_spec_, s);
    CUFFT_CHECK(cufftExecZ2D(plan_inv_, reinterpret_cast<cufftDoubleComplex*>(spec_), grid_));
    dev::launch_interp(nufft_, s);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[3], s));
    dev::launch_finalize(pot_sorted_, far_sorted_, trg_, trg_perm_, q, pot, n_, s);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[4], s));
    PDMK_CUDA_CHECK(cudaGetLastError());
}

StageTimes DeviceTree::last_times() {
    StageTimes t;
    PDMK_CUDA_CHECK(cudaEventSynchronize(ev_[4]));
    float t01, t12, t23, t34;
    PDMK_CUDA_CHECK(cudaEventElapsedTime(&t01, ev_[0], ev_[1]));
    PDMK_CUDA_CHECK(cudaEventElapsedTime(&t12, ev_[1], ev_[2]));
    PDMK_CUDA_CHECK(cudaEventElapsedTime(&t23, ev_[2], ev_[3]));
    PDMK_CUDA_CHECK(cudaEventElapsedTime(&t34, ev_[3], ev_[4]));
    t.dmk_ms = t01;
    t.direct_ms = t12 + t34;
    t.nufft_ms = t23;
    t.near_ms = t12;
    t.finalize_ms = t34;
    return t;
}

void DeviceTree::evaluate_device(const double* q_user_d, double* pot_user_d, StageTimes* times) {
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    last_was_multi_ = false;
    run(q_user_d, pot_user_d);
    if (times) *times = last_times();
}

void DeviceTree::evaluate_parts_host(const double* q_user, double* tree_part, double* far_part) {
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    PDMK_CUDA_CHECK(cudaMemcpyAsync(q_dev_, q_user, sizeof(double) * n_, cudaMemcpyHostToDevice, stream_));
    run(q_dev_, pot_dev_);
    double* tp = nullptr;
    double* fp = nullptr;
    PDMK_CUDA_CHECK(cudaMallocAsync(&tp, sizeof(double) * n_, stream_));
    PDMK_CUDA_CHECK(cudaMallocAsync(&fp, sizeof(double) * n_, stream_));
    dev::launch_desort_parts(pot_sorted_, far_sorted_, trg_, trg_perm_, q_dev_, tp, fp, n_, stream_);
    PDMK_CUDA_CHECK(cudaMemcpyAsync(tree_part, tp, sizeof(double) * n_, cudaMemcpyDeviceToHost, stream_));
    PDMK_CUDA_CHECK(cudaMemcpyAsync(far_part, fp, sizeof(double) * n_, cudaMemcpyDeviceToHost, stream_));
    PDMK_CUDA_CHECK(cudaFreeAsync(tp, stream_));
    PDMK_CUDA_CHECK(cudaFreeAsync(fp, stream_));
    PDMK_CUDA_CHECK(cudaStreamSynchronize(stream_));
}

void DeviceTree::ensure_grad() {
    if (grad_sorted_) return;
    ensure_fp64_working_set();
    grad_sorted_ = alloc<double>(3 * (size_t)n_);
    far_grad_ = alloc<double>(3 * (size_t)n_);
    grad_dev_ = alloc<double>(3 * (size_t)n_);
    spec_save_ = alloc<dev::cd>(n_spec_);
    spec_tmp_ = alloc<dev::cd>(n_spec_);
}

void DeviceTree::evaluate_grad_device(const double* q, double* pot, double* grad) {
    require_periodic("evaluate_grad");
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    last_was_multi_ = false;
    ensure_grad();
    struct Flag {  // the leaf-evaluation gradients run only inside this call
        bool& f;
        explicit Flag(bool& x) : f(x) { f = true; }
        ~Flag() { f = false; }
    } on(grad_on_);
    cudaStream_t s = stream_;
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[0], s));
    PDMK_CUDA_CHECK(cudaMemsetAsync(pot_sorted_, 0, sizeof(double) * n_, s));
    PDMK_CUDA_CHECK(cudaMemsetAsync(grad_sorted_, 0, sizeof(double) * 3 * (size_t)n_, s));
    run_fp64_tree(q, f64_scratch_, f64_scratch_elems_, s);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[1], s));
    dev::launch_near_pg(near_, grad_sorted_, n_, s);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[2], s));
    // far field: potential, then the three spectral derivatives of the same spectrum
    dev::launch_nufft_gather_q(trg_perm_, q, q_sorted_, n_, s);
    PDMK_CUDA_CHECK(cudaMemsetAsync(grid_, 0, sizeof(double) * n_grid_, s));
    dev::launch_spread(nufft_, nufft_max_jk_, nufft_max_ex_, s);
    CUFFT_CHECK(cufftExecD2Z(plan_fwd_, grid_, reinterpret_cast<cufftDoubleComplex*>(spec_)));
    dev::launch_multiply(spec_, mult_, n_spec_, s);
    // the complex-to-real transform overwrites its input: keep a copy
    PDMK_CUDA_CHECK(cudaMemcpyAsync(spec_save_, spec_, sizeof(dev::cd) * n_spec_, cudaMemcpyDeviceToDevice, s));
    CUFFT_CHECK(cufftExecZ2D(plan_inv_, reinterpret_cast<cufftDoubleComplex*>(spec_), grid_));
    dev::launch_interp(nufft_, s);
    for (int d = 0; d < 3; ++d) {
        dev::launch_grad_multiply(spec_save_, spec_tmp_, nufft_.n1, nufft_.n2, nufft_.n3, d, frame_, s);
        CUFFT_CHECK(cufftExecZ2D(plan_inv_, reinterpret_cast<cufftDoubleComplex*>(spec_tmp_), grid_));
        dev::NufftArgs na = nufft_;
        na.far = far_grad_ + (int64_t)d * n_;
        dev::launch_interp(na, s);
    }
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[3], s));
    dev::launch_finalize(pot_sorted_, far_sorted_, trg_, trg_perm_, q, pot, n_, s);
    dev::launch_finalize_grad(grad_sorted_, far_grad_, trg_perm_, grad, n_, frame_, s);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[4], s));
    PDMK_CUDA_CHECK(cudaGetLastError());
    PDMK_CUDA_CHECK(cudaStreamSynchronize(s));
}

void DeviceTree::evaluate_grad_host(const double* q_user, double* pot_user, double* grad_user) {
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    ensure_grad();
    PDMK_CUDA_CHECK(cudaMemcpyAsync(q_dev_, q_user, sizeof(double) * n_, cudaMemcpyHostToDevice, stream_));
    evaluate_grad_device(q_dev_, pot_dev_, grad_dev_);
    PDMK_CUDA_CHECK(cudaMemcpyAsync(pot_user, pot_dev_, sizeof(double) * n_, cudaMemcpyDeviceToHost, stream_));
    PDMK_CUDA_CHECK(cudaMemcpyAsync(grad_user, grad_dev_, sizeof(double) * 3 * (size_t)n_, cudaMemcpyDeviceToHost,
                                    stream_));
    PDMK_CUDA_CHECK(cudaStreamSynchronize(stream_));
}

void DeviceTree::evaluate_host(const double* q_user, double* pot_user, StageTimes* times) {
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    PDMK_CUDA_CHECK(cudaMemcpyAsync(q_dev_, q_user, sizeof(double) * n_, cudaMemcpyHostToDevice, stream_));
    evaluate_device(q_dev_, pot_dev_, times);
    PDMK_CUDA_CHECK(cudaMemcpyAsync(pot_user, pot_dev_, sizeof(double) * n_, cudaMemcpyDeviceToHost, stream_));
    PDMK_CUDA_CHECK(cudaStreamSynchronize(stream_));
}

}  // namespace pdmkb
