// ORACLE — test infrastructure only.  Nothing in the product links, imports or
// calls this file; only tests/, the smoke check and the CPU-baseline leg of
// bench.py load it, as the checker.
//
// A CPU restatement (FP64, OpenMP) of the reference's evaluate path for one
// periodic tree, written as plain per-box loops that follow the reference's
// stage structure:
//   charge gather + sort                cpp/src/periodic_dmk.cpp:164-169, cpp/src/dmk/pbc_tree.cpp:1807-1821
//   upward: charge -> proxy moments     cpp/src/dmk/pbc_tree.cpp:1152-1163, cpp/src/dmk/proxy.cpp:153-212
//   upward: child -> parent (c2p)       cpp/src/dmk/pbc_tree.cpp:1166-1185, cpp/src/dmk/tensorprod.cpp:39-75
//   outgoing plane waves                cpp/src/dmk/pbc_tree.cpp:1208-1249, cpp/src/dmk/proxy.cpp:42-90
//   shift + pw -> proxy + p2c + eval    cpp/src/dmk/pbc_tree.cpp:1251-1440, cpp/src/dmk/planewave.cpp:49-105,
//                                       cpp/src/dmk/proxy.cpp:307-448
//   residual near field                 cpp/src/dmk/pbc_tree.cpp:1442-1681, cpp/include/dmk/vector_kernels.hpp:354-421
//   self correction + desort            cpp/src/dmk/pbc_tree.cpp:1759-1805
//   periodic far field                  cpp/src/dmk/pbc.cpp:359-541
// Differences from the reference, both exact up to rounding:
//   * the far field is the exact reciprocal-lattice sum over the same modes and
//     weights (the reference uses a NUFFT at tolerance eps/4);
//   * the near field masks pairs by distance instead of culling them by box
//     contact geometry first (culled pairs all have r >= b and contribute 0).
// The tree, lists and tables come from the host plan builder; the tree and
// lists are checked box for box against the oracle's own independent builder
// (oracle_tree.cpp, tests/test_oracle_pins.py), the tables end to end against
// the Ewald sums below and against the reference's own PSWF / quadrature /
// image code (golden fixtures).
//
// Also: a direct O(N^2) Ewald sum (cpp/src/ewald_nufft.cpp:777-910) as the
// independent physics check.
#include <omp.h>

#include <array>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include "../periodicdmk_b200/csrc/host/plan.hpp"
#include "../periodicdmk_b200/csrc/host/pswf.hpp"

using pdmkb::cplx;
using pdmkb::Plan;

namespace {

// out(a,b,c) (+)= sum_{ijk} Ux(a,i) Uy(b,j) Uz(c,k) in(i,j,k), x fastest.
// U_d(a,i) = m[d][a + no*i] (column-major no x ni).
template <typename Tin, typename Tm, typename Tout>
void separable(int ni, int no, const Tin* in, const Tm* mx, const Tm* my, const Tm* mz, Tout* out) {
    using T = decltype(Tin() * Tm());
    std::vector<T> t1((size_t)no * ni * ni), t2((size_t)no * no * ni);
    for (int k = 0; k < ni; ++k)
        for (int j = 0; j < ni; ++j)
            for (int a = 0; a < no; ++a) {
                T s = T(0);
                for (int i = 0; i < ni; ++i) s += mx[a + (size_t)no * i] * in[i + (size_t)ni * (j + (size_t)ni * k)];
                t1[a + (size_t)no * (j + (size_t)ni * k)] = s;
            }
    for (int k = 0; k < ni; ++k)
        for (int b = 0; b < no; ++b)
            for (int a = 0; a < no; ++a) {
                T s = T(0);
                for (int j = 0; j < ni; ++j) s += my[b + (size_t)no * j] * t1[a + (size_t)no * (j + (size_t)ni * k)];
                t2[a + (size_t)no * (b + (size_t)no * k)] = s;
            }
    for (int c = 0; c < no; ++c)
        for (int b = 0; b < no; ++b)
            for (int a = 0; a < no; ++a) {
                T s = T(0);
                for (int k = 0; k < ni; ++k) s += mz[c + (size_t)no * k] * t2[a + (size_t)no * (b + (size_t)no * k)];
                out[a + (size_t)no * (b + (size_t)no * c)] += s;
            }
}

void cheb(int p, double x, double* t) {
    t[0] = 1.0;
    if (p > 1) t[1] = x;
    for (int a = 2; a < p; ++a) t[a] = 2.0 * x * t[a - 1] - t[a - 2];
}

struct Components {
    std::vector<double> near, mid, self, far;  // user order
};

void far_nufft(const Plan& P, const double* q_user, std::vector<double>& far);

void oracle_eval(const Plan& P, const double* q_user, Components& C, bool do_far, bool fast_far) {
    const int p = P.p, n = P.n_pw, n2 = P.n_pw2, M = P.n_modes;
    const size_t ncoef = (size_t)p * p * p;
    const int N = P.n_src;
    std::vector<double> qs(P.n_all);
    for (int i = 0; i < P.n_all; ++i) qs[i] = q_user[P.src_charge_idx[i]];

    // ---- upward: proxy moments
    std::vector<double> up((size_t)P.n_proxy_up * ncoef, 0.0);
    {
        // group work by centre box so each centre is written by one thread
        std::vector<std::vector<int>> by_center(P.nboxes);
        for (int w = 0; w < (int)P.c2proxy_work.size(); ++w) by_center[P.c2proxy_work[w].center_box].push_back(w);
        std::vector<int> centers;
        for (int b = 0; b < P.nboxes; ++b)
            if (!by_center[b].empty()) centers.push_back(b);
#pragma omp parallel for schedule(dynamic)
        for (int ci = 0; ci < (int)centers.size(); ++ci) {
            const int cb = centers[ci];
            double* M3 = &up[P.proxy_up_off[cb]];
            std::vector<double> tx(p), ty(p), tz(p);
            for (int w : by_center[cb]) {
                const auto& W = P.c2proxy_work[w];
                const double sc = 2.0 / P.boxsize[W.level];
                const double* c = &P.centers[3 * cb];
                for (int s = P.src_start[W.src_box]; s < P.src_start[W.src_box] + P.src_count[W.src_box]; ++s) {
                    const double* x = &P.src_sorted[3 * (size_t)s];
                    cheb(p, sc * (x[0] - c[0]), tx.data());
                    cheb(p, sc * (x[1] - c[1]), ty.data());
                    cheb(p, sc * (x[2] - c[2]), tz.data());
                    for (int k = 0; k < p; ++k)
                        for (int j = 0; j < p; ++j) {
                            const double f = qs[s] * ty[j] * tz[k];
                            double* row = M3 + (size_t)p * (j + (size_t)p * k);
                            for (int i = 0; i < p; ++i) row[i] += f * tx[i];
                        }
                }
            }
        }
    }
    // ---- upward: children -> parent, bottom-up
    {
        std::vector<double> c2p((size_t)8 * 3 * p * p);
        for (int c = 0; c < 8; ++c)
            for (int d = 0; d < 3; ++d)
                for (int a = 0; a < p; ++a)
                    for (int i = 0; i < p; ++i)
                        c2p[((size_t)c * 3 + d) * p * p + a + (size_t)p * i] =
                            P.p2c[((size_t)c * 3 + d) * p * p + i + (size_t)p * a];
        for (int l = P.nlevels - 1; l >= 0; --l) {
            const auto& LB = P.level_boxes[l];
#pragma omp parallel for schedule(dynamic)
            for (int bi = 0; bi < (int)LB.size(); ++bi) {
                const int b = LB[bi];
                if (!P.has_proxy_from_children[b]) continue;
                for (int c = 0; c < 8; ++c) {
                    const int ch = P.children[b][c];
                    if (ch < 0 || !(P.src_count[ch] > 0 && P.ifpwexp[ch])) continue;
                    const double* m = &c2p[(size_t)c * 3 * p * p];
                    separable<double, double, double>(p, p, &up[P.proxy_up_off[ch]], m, m + p * p, m + 2 * p * p,
                                                      &up[P.proxy_up_off[b]]);
                }
            }
        }
    }
    // ---- outgoing plane waves
    std::vector<cplx> pw((size_t)P.n_pw_exp * M, cplx(0));
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < P.nboxes; ++b) {
        if (P.pw_off[b] < 0) continue;
        const auto& T = P.lev[P.depth[b]];
        // out(k1,k2,k3) = sum poly2pw(k1,m1) poly2pw(k2,m2) poly2pw(k3,m3) proxy(m1,m2,m3),
        // k3 restricted to the half-space (first n2 z-frequencies).
        {
            const double* in = &up[P.proxy_up_off[b]];
            std::vector<cplx> t1((size_t)n * p * p), t2((size_t)n * n * p);
            for (int k = 0; k < p; ++k)
                for (int j = 0; j < p; ++j)
                    for (int a = 0; a < n; ++a) {
                        cplx s(0);
                        for (int i = 0; i < p; ++i) s += T.poly2pw[a + (size_t)n * i] * in[i + (size_t)p * (j + (size_t)p * k)];
                        t1[a + (size_t)n * (j + (size_t)p * k)] = s;
                    }
            for (int k = 0; k < p; ++k)
                for (int bb = 0; bb < n; ++bb)
                    for (int a = 0; a < n; ++a) {
                        cplx s(0);
                        for (int j = 0; j < p; ++j) s += T.poly2pw[bb + (size_t)n * j] * t1[a + (size_t)n * (j + (size_t)p * k)];
                        t2[a + (size_t)n * (bb + (size_t)n * k)] = s;
                    }
            cplx* out = &pw[P.pw_off[b]];
            for (int c = 0; c < n2; ++c)
                for (int bb = 0; bb < n; ++bb)
                    for (int a = 0; a < n; ++a) {
                        cplx s(0);
                        for (int k = 0; k < p; ++k) s += T.poly2pw[c + (size_t)n * k] * t2[a + (size_t)n * (bb + (size_t)n * k)];
                        out[a + (size_t)n * (bb + (size_t)n * c)] = s;
                    }
        }
    }
    // ---- downward: per level, shift + pw->proxy + parent->child
    std::vector<double> down((size_t)P.n_proxy_down * ncoef, 0.0);
    for (int l = 0; l < P.nlevels; ++l) {
        const auto& T = P.lev[l];
        const double bs = P.boxsize[l];
        const auto& LB = P.level_boxes[l];
#pragma omp parallel for schedule(dynamic)
        for (int bi = 0; bi < (int)LB.size(); ++bi) {
            const int b = LB[bi];
            const bool has_output = P.trg_count[b] > 0;
            if (!(P.ifpwexp[b] && P.src_count[b] + P.trg_count[b] > 0 && has_output)) continue;
            std::vector<cplx> pin((size_t)M, cplx(0));
            // self term (stencil 13) then colleagues
            auto add_shift = [&](int src_box, int st) {
                const cplx* po = &pw[P.pw_off[src_box]];
                const double* re = &T.shift[(size_t)st * 2 * M];
                const double* im = re + M;
                for (int m = 0; m < M; ++m) pin[m] += po[m] * cplx(re[m], im[m]);
            };
            add_shift(b, 13);
            for (int ind = 0; ind < 27; ++ind) {
                const int nb = P.colleagues[b][ind];
                if (nb < 0 || nb == b) continue;
                if (P.is_leaf[b] && P.is_leaf[nb]) continue;
                if (P.pw_off[nb] < 0) continue;
                int st = 0, stride = 1;
                for (int d = 0; d < 3; ++d) {
                    const int kd = (int)std::lround((P.centers[3 * b + d] - P.centers[3 * nb + d]) / bs) + 1;
                    st += kd * stride;
                    stride *= 3;
                }
                add_shift(nb, st);
            }
            // proxy_down += 2 Re sum pw2poly(m1,a) pw2poly(m2,b) w(m3) pw2poly(m3,c) pin(m1,m2,m3)
            std::vector<cplx> t1((size_t)p * n * n2), t2((size_t)p * p * n2);
            for (int m3 = 0; m3 < n2; ++m3)
                for (int m2 = 0; m2 < n; ++m2)
                    for (int a = 0; a < p; ++a) {
                        cplx s(0);
                        for (int m1 = 0; m1 < n; ++m1) s += T.pw2poly[m1 + (size_t)n * a] * pin[m1 + (size_t)n * (m2 + (size_t)n * m3)];
                        t1[a + (size_t)p * (m2 + (size_t)n * m3)] = s;
                    }
            for (int m3 = 0; m3 < n2; ++m3)
                for (int bb = 0; bb < p; ++bb)
                    for (int a = 0; a < p; ++a) {
                        cplx s(0);
                        for (int m2 = 0; m2 < n; ++m2) s += T.pw2poly[m2 + (size_t)n * bb] * t1[a + (size_t)p * (m2 + (size_t)n * m3)];
                        t2[a + (size_t)p * (bb + (size_t)p * m3)] = s;
                    }
            double* dn = &down[P.proxy_down_off[b]];
            for (int c = 0; c < p; ++c)
                for (int bb = 0; bb < p; ++bb)
                    for (int a = 0; a < p; ++a) {
                        cplx s(0);
                        for (int m3 = 0; m3 < n2; ++m3) {
                            const double w = m3 >= n / 2 ? 0.5 : 1.0;
                            s += w * T.pw2poly[m3 + (size_t)n * c] * t2[a + (size_t)p * (bb + (size_t)p * m3)];
                        }
                        dn[a + (size_t)p * (bb + (size_t)p * c)] += 2.0 * s.real();
                    }
            if (!P.iftensprodeval[b]) {
                for (int c = 0; c < 8; ++c) {
                    const int ch = P.children[b][c];
                    if (ch < 0 || !(P.src_count[ch] + P.trg_count[ch])) continue;
                    const double* m = &P.p2c[(size_t)c * 3 * p * p];
                    separable<double, double, double>(p, p, dn, m, m + p * p, m + 2 * p * p, &down[P.proxy_down_off[ch]]);
                }
            }
        }
    }
    // ---- proxy -> targets at leaves
    std::vector<double> mid_sorted(N, 0.0), near_sorted(N, 0.0);
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < P.nboxes; ++b) {
        if (!P.iftensprodeval[b] || P.trg_count[b] == 0) continue;
        const double sc = 2.0 / P.boxsize[P.depth[b]];
        const double* c = &P.centers[3 * b];
        const double* cf = &down[P.proxy_down_off[b]];
        std::vector<double> tx(p), ty(p), tz(p);
        for (int t = P.trg_start[b]; t < P.trg_start[b] + P.trg_count[b]; ++t) {
            const double* x = &P.trg_sorted[3 * (size_t)t];
            cheb(p, sc * (x[0] - c[0]), tx.data());
            cheb(p, sc * (x[1] - c[1]), ty.data());
            cheb(p, sc * (x[2] - c[2]), tz.data());
            double s = 0;
            for (int k = 0; k < p; ++k)
                for (int j = 0; j < p; ++j) {
                    double r = 0;
                    const double* row = cf + (size_t)p * (j + (size_t)p * k);
                    for (int i = 0; i < p; ++i) r += row[i] * tx[i];
                    s += r * ty[j] * tz[k];
                }
            mid_sorted[t] += s;
        }
    }
    // ---- residual near field
    const std::vector<double>& cf = P.resid;
    const int nc = (int)cf.size();
#pragma omp parallel for schedule(dynamic)
    for (int wi = 0; wi < (int)P.direct_work.size(); ++wi) {
        const int tb = P.direct_work[wi];
        if (P.trg_count[tb] == 0) continue;
        const int tl = P.depth[tb];
        for (int li = P.list1_start[tb]; li < P.list1_start[tb + 1]; ++li) {
            const int sb = P.list1[li];
            int sl = P.depth[sb];
            double bsize = P.boxsize[sl];
            if (P.ifpwexp[sb] && sb == tb)
                bsize /= 2.0;
            else if (sl < tl)
                bsize = P.boxsize[tl];
            const double d2max = bsize * bsize, rsc = 2.0 / bsize, cen = -bsize / 2.0;
            for (int t = P.trg_start[tb]; t < P.trg_start[tb] + P.trg_count[tb]; ++t) {
                const double* x = &P.trg_sorted[3 * (size_t)t];
                double acc = 0;
                for (int s = P.src_start[sb]; s < P.src_start[sb] + P.src_count[sb]; ++s) {
                    const double* y = &P.src_sorted[3 * (size_t)s];
                    const double dx = x[0] - y[0], dy = x[1] - y[1], dz = x[2] - y[2];
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    if (!(r2 > 1e-30 && r2 < d2max)) continue;
                    const double r = std::sqrt(r2);
                    const double xm = (r + cen) * rsc;
                    double pv = cf[nc - 1];
                    for (int i = nc - 2; i >= 0; --i) pv = pv * xm + cf[i];
                    acc += qs[s] * pv / r;
                }
                near_sorted[t] += acc;
            }
        }
    }
    // ---- self correction and desort
    C.near.assign(N, 0.0);
    C.mid.assign(N, 0.0);
    C.self.assign(N, 0.0);
    C.far.assign(N, 0.0);
    for (int b = 0; b < P.nboxes; ++b) {
        if (!P.is_leaf[b] || P.trg_count[b] == 0) continue;
        const double w0 = P.w0[P.depth[b] + P.ifpwexp[b]];
        for (int t = P.trg_start[b]; t < P.trg_start[b] + P.trg_count[b]; ++t) {
            const int u = P.trg_perm[t];
            C.self[u] = -w0 * q_user[u];
            C.near[u] = near_sorted[t];
            C.mid[u] = mid_sorted[t];
        }
    }
    if (!do_far) return;
    if (fast_far) {
        far_nufft(P, q_user, C.far);
        return;
    }
    // ---- far field: exact sum over the (ms, mt, mu) modes with nonzero weight
    const double twopi = 2.0 * M_PI;
    std::vector<double> X(N), Y(N), Z(N);
    for (int i = 0; i < N; ++i) {
        const double* r = &P.r_user[3 * (size_t)i];
        X[i] = twopi * (P.umatinv[0] * r[0] + P.umatinv[3] * r[1] + P.umatinv[6] * r[2]);
        Y[i] = twopi * (P.umatinv[4] * r[1] + P.umatinv[7] * r[2]);
        Z[i] = twopi * (P.umatinv[8] * r[2]);
    }
    struct Mode {
        int i, j, k;
        double w;
    };
    std::vector<Mode> modes;
    {
        size_t idx = 0;
        for (int k = -P.mu / 2; k <= (P.mu - 1) / 2; ++k)
            for (int j = -P.mt / 2; j <= (P.mt - 1) / 2; ++j)
                for (int i = -P.ms / 2; i <= (P.ms - 1) / 2; ++i, ++idx)
                    if (P.ff_weights[idx] != 0.0) modes.push_back({i, j, k, P.ff_weights[idx]});
    }
    const int nm = (int)modes.size();
    std::vector<cplx> S(nm, cplx(0));
#pragma omp parallel for schedule(static)
    for (int m = 0; m < nm; ++m) {
        cplx s(0);
        for (int l = 0; l < N; ++l) {
            const double ph = modes[m].i * X[l] + modes[m].j * Y[l] + modes[m].k * Z[l];
            s += q_user[l] * cplx(std::cos(ph), -std::sin(ph));
        }
        S[m] = s * modes[m].w;
    }
#pragma omp parallel for schedule(static)
    for (int l = 0; l < N; ++l) {
        double u = 0;
        for (int m = 0; m < nm; ++m) {
            const double ph = modes[m].i * X[l] + modes[m].j * Y[l] + modes[m].k * Z[l];
            u += S[m].real() * std::cos(ph) - S[m].imag() * std::sin(ph);
        }
        C.far[l] = u;
    }
}

// Far field by a CPU NUFFT (for the CPU timing baseline only; the exact sum
// above is the parity reference).  Exponential-of-semicircle kernel
// phi(z) = exp(b (sqrt(1 - z^2) - 1)), width W, b = 2.30 W, 2x oversampled
// grid; the small grid is transformed to and from the mode box by separable
// direct DFTs.
void far_nufft(const Plan& P, const double* q, std::vector<double>& far) {
    const int N = P.n_src;
    int W = (int)std::ceil(-std::log10(P.dp.eps / 4.0)) + 1;
    W = std::min(14, std::max(4, W));
    const double beta = 2.30 * W;
    const int m[3] = {P.ms, P.mt, P.mu};
    int ng[3];
    for (int d = 0; d < 3; ++d) ng[d] = std::max(2 * m[d], 2 * W) + (std::max(2 * m[d], 2 * W) & 1);
    const double twopi = 2.0 * M_PI;
    const size_t G = (size_t)ng[0] * ng[1] * ng[2];
    auto kern = [&](double z) { return z * z < 1.0 ? std::exp(beta * (std::sqrt(1.0 - z * z) - 1.0)) : 0.0; };
    std::vector<std::array<int, 3>> l0(N);
    std::vector<double> kv((size_t)N * 3 * W);
    for (int i = 0; i < N; ++i) {
        const double* r = &P.r_user[3 * (size_t)i];
        const double s[3] = {P.umatinv[0] * r[0] + P.umatinv[3] * r[1] + P.umatinv[6] * r[2],
                             P.umatinv[4] * r[1] + P.umatinv[7] * r[2], P.umatinv[8] * r[2]};
        for (int d = 0; d < 3; ++d) {
            const double t = (s[d] - std::floor(s[d])) * ng[d];
            l0[i][d] = (int)std::ceil(t - 0.5 * W);
            for (int a = 0; a < W; ++a) kv[((size_t)i * 3 + d) * W + a] = kern((t - (l0[i][d] + a)) / (0.5 * W));
        }
    }
    auto wrap = [](int i, int n) { i %= n; return i < 0 ? i + n : i; };
    // spread (per-thread grids, then reduce)
    std::vector<double> grid(G, 0.0);
#pragma omp parallel
    {
        std::vector<double> g(G, 0.0);
#pragma omp for schedule(static)
        for (int i = 0; i < N; ++i) {
            const double* kx = &kv[((size_t)i * 3 + 0) * W];
            const double* ky = &kv[((size_t)i * 3 + 1) * W];
            const double* kz = &kv[((size_t)i * 3 + 2) * W];
            for (int a = 0; a < W; ++a) {
                const size_t ia = (size_t)wrap(l0[i][0] + a, ng[0]) * ng[1];
                for (int b = 0; b < W; ++b) {
                    const size_t ib = (ia + wrap(l0[i][1] + b, ng[1])) * ng[2];
                    const double f = q[i] * kx[a] * ky[b];
                    for (int c = 0; c < W; ++c) g[ib + wrap(l0[i][2] + c, ng[2])] += f * kz[c];
                }
            }
        }
#pragma omp critical
        for (size_t k = 0; k < G; ++k) grid[k] += g[k];
    }
    // kernel Fourier transforms on each axis
    std::vector<double> gx(200), gw(200);
    pdmkb::gauss_legendre(200, gx.data(), gw.data());
    auto phihat = [&](int d, int k) {
        const double alpha = 0.5 * W * twopi / ng[d];
        double s = 0;
        for (int i = 0; i < 200; ++i) s += gw[i] * kern(gx[i]) * std::cos(k * alpha * gx[i]);
        return alpha * s;
    };
    // forward separable DFT: grid (l1,l2,l3) -> B(k1,k2,k3) for k_d in [-m_d/2, (m_d-1)/2]
    std::vector<cplx> e[3];
    for (int d = 0; d < 3; ++d) {
        e[d].resize((size_t)m[d] * ng[d]);
        for (int k = 0; k < m[d]; ++k)
            for (int l = 0; l < ng[d]; ++l) {
                const double ph = -twopi * (double)(k - m[d] / 2) * l / ng[d];
                e[d][(size_t)k * ng[d] + l] = cplx(std::cos(ph), std::sin(ph));
            }
    }
    // layout grid[(l1*n2 + l2)*n3 + l3]
    std::vector<cplx> b1((size_t)m[0] * ng[1] * ng[2]), b2((size_t)m[0] * m[1] * ng[2]), b3((size_t)m[0] * m[1] * m[2]);
#pragma omp parallel for collapse(2)
    for (int k1 = 0; k1 < m[0]; ++k1)
        for (int l2 = 0; l2 < ng[1]; ++l2)
            for (int l3 = 0; l3 < ng[2]; ++l3) {
                cplx s(0);
                for (int l1 = 0; l1 < ng[0]; ++l1) s += e[0][(size_t)k1 * ng[0] + l1] * grid[((size_t)l1 * ng[1] + l2) * ng[2] + l3];
                b1[((size_t)k1 * ng[1] + l2) * ng[2] + l3] = s;
            }
#pragma omp parallel for collapse(2)
    for (int k1 = 0; k1 < m[0]; ++k1)
        for (int k2 = 0; k2 < m[1]; ++k2)
            for (int l3 = 0; l3 < ng[2]; ++l3) {
                cplx s(0);
                for (int l2 = 0; l2 < ng[1]; ++l2) s += e[1][(size_t)k2 * ng[1] + l2] * b1[((size_t)k1 * ng[1] + l2) * ng[2] + l3];
                b2[((size_t)k1 * m[1] + k2) * ng[2] + l3] = s;
            }
    const double H = twopi * twopi * twopi / ((double)ng[0] * ng[1] * ng[2]);
    std::vector<double> ph[3];
    for (int d = 0; d < 3; ++d) {
        ph[d].resize(m[d]);
        for (int k = 0; k < m[d]; ++k) ph[d][k] = phihat(d, k - m[d] / 2);
    }
#pragma omp parallel for collapse(2)
    for (int k1 = 0; k1 < m[0]; ++k1)
        for (int k2 = 0; k2 < m[1]; ++k2)
            for (int k3 = 0; k3 < m[2]; ++k3) {
                cplx s(0);
                for (int l3 = 0; l3 < ng[2]; ++l3) s += e[2][(size_t)k3 * ng[2] + l3] * b2[((size_t)k1 * m[1] + k2) * ng[2] + l3];
                // ff_weights layout: k3 slowest, k1 fastest
                const double w = P.ff_weights[((size_t)k3 * m[1] + k2) * m[0] + k1];
                const double Ps = ph[0][k1] * ph[1][k2] * ph[2][k3];
                b3[((size_t)k1 * m[1] + k2) * m[2] + k3] = s * (w * H * H / (Ps * Ps));
            }
    // inverse separable DFT back to the grid (real part)
#pragma omp parallel for collapse(2)
    for (int k1 = 0; k1 < m[0]; ++k1)
        for (int k2 = 0; k2 < m[1]; ++k2)
            for (int l3 = 0; l3 < ng[2]; ++l3) {
                cplx s(0);
                for (int k3 = 0; k3 < m[2]; ++k3) s += std::conj(e[2][(size_t)k3 * ng[2] + l3]) * b3[((size_t)k1 * m[1] + k2) * m[2] + k3];
                b2[((size_t)k1 * m[1] + k2) * ng[2] + l3] = s;
            }
#pragma omp parallel for collapse(2)
    for (int k1 = 0; k1 < m[0]; ++k1)
        for (int l2 = 0; l2 < ng[1]; ++l2)
            for (int l3 = 0; l3 < ng[2]; ++l3) {
                cplx s(0);
                for (int k2 = 0; k2 < m[1]; ++k2) s += std::conj(e[1][(size_t)k2 * ng[1] + l2]) * b2[((size_t)k1 * m[1] + k2) * ng[2] + l3];
                b1[((size_t)k1 * ng[1] + l2) * ng[2] + l3] = s;
            }
#pragma omp parallel for collapse(2)
    for (int l1 = 0; l1 < ng[0]; ++l1)
        for (int l2 = 0; l2 < ng[1]; ++l2)
            for (int l3 = 0; l3 < ng[2]; ++l3) {
                cplx s(0);
                for (int k1 = 0; k1 < m[0]; ++k1) s += std::conj(e[0][(size_t)k1 * ng[0] + l1]) * b1[((size_t)k1 * ng[1] + l2) * ng[2] + l3];
                grid[((size_t)l1 * ng[1] + l2) * ng[2] + l3] = s.real();
            }
    far.assign(N, 0.0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        const double* kx = &kv[((size_t)i * 3 + 0) * W];
        const double* ky = &kv[((size_t)i * 3 + 1) * W];
        const double* kz = &kv[((size_t)i * 3 + 2) * W];
        double u = 0;
        for (int a = 0; a < W; ++a) {
            const size_t ia = (size_t)wrap(l0[i][0] + a, ng[0]) * ng[1];
            for (int b = 0; b < W; ++b) {
                const size_t ib = (ia + wrap(l0[i][1] + b, ng[1])) * ng[2];
                double sc = 0;
                for (int c = 0; c < W; ++c) sc += kz[c] * grid[ib + wrap(l0[i][2] + c, ng[2])];
                u += kx[a] * ky[b] * sc;
            }
        }
        far[i] = u;
    }
}

}  // namespace

extern "C" {

int oracle_evaluate2(const double* cell, int n, const double* pos, const double* q, int n_digits, int n_per_leaf,
                     int nz, int with_far, int fast_far, double* pot, double* comp);

// Evaluate potentials with the oracle.  comp (optional, 4*N): near | mid | self | far.
// Returns 0 on success, -1 on error (message on stderr).
int oracle_evaluate(const double* cell, int n, const double* pos, const double* q, int n_digits, int n_per_leaf,
                    int nz, int with_far, double* pot, double* comp) {
    return oracle_evaluate2(cell, n, pos, q, n_digits, n_per_leaf, nz, with_far, 0, pot, comp);
}

// with_far: 0 none, 1 far field; fast_far: 0 exact reciprocal sum, 1 CPU NUFFT.
int oracle_evaluate2(const double* cell, int n, const double* pos, const double* q, int n_digits, int n_per_leaf,
                     int nz, int with_far, int fast_far, double* pot, double* comp) {
    try {
        Plan P = pdmkb::build_plan(cell, n, pos, n_digits, n_per_leaf, nz);
        Components C;
        oracle_eval(P, q, C, with_far != 0, fast_far != 0);
        for (int i = 0; i < n; ++i) pot[i] = C.near[i] + C.mid[i] + C.self[i] + C.far[i];
        if (comp) {
            std::memcpy(comp, C.near.data(), n * sizeof(double));
            std::memcpy(comp + n, C.mid.data(), n * sizeof(double));
            std::memcpy(comp + 2 * (size_t)n, C.self.data(), n * sizeof(double));
            std::memcpy(comp + 3 * (size_t)n, C.far.data(), n * sizeof(double));
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle_evaluate: %s\n", e.what());
        return -1;
    }
}

// Build-once / evaluate-many form (for timing the evaluate alone, as the
// reference's PeriodicDMKTreeT separates construction from evaluate).
void* oracle_plan_new(const double* cell, int n, const double* pos, int n_digits, int n_per_leaf, int nz) {
    try {
        return new Plan(pdmkb::build_plan(cell, n, pos, n_digits, n_per_leaf, nz));
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle_plan_new: %s\n", e.what());
        return nullptr;
    }
}

int oracle_plan_eval(void* h, const double* q, int with_far, int fast_far, double* pot) {
    try {
        const Plan& P = *static_cast<Plan*>(h);
        Components C;
        oracle_eval(P, q, C, with_far != 0, fast_far != 0);
        for (int i = 0; i < P.n_src; ++i) pot[i] = C.near[i] + C.mid[i] + C.self[i] + C.far[i];
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle_plan_eval: %s\n", e.what());
        return -1;
    }
}

void oracle_plan_free(void* h) { delete static_cast<Plan*>(h); }

// Plan statistics for tests: out[0..9] = n_all, nboxes, nlevels, n_target_leaves,
// n_pw_boxes, n_c2proxy_work, list1 total, ms, mt, mu.
int oracle_plan_stats(const double* cell, int n, const double* pos, int n_digits, int n_per_leaf, int nz,
                      long long* out) {
    try {
        Plan P = pdmkb::build_plan(cell, n, pos, n_digits, n_per_leaf, nz);
        int nlt = 0;
        for (int b = 0; b < P.nboxes; ++b)
            if (P.is_leaf[b] && P.trg_count[b] > 0) nlt++;
        out[0] = P.n_all;
        out[1] = P.nboxes;
        out[2] = P.nlevels;
        out[3] = nlt;
        out[4] = P.n_pw_exp;
        out[5] = (long long)P.c2proxy_work.size();
        out[6] = (long long)P.list1.size();
        out[7] = P.ms;
        out[8] = P.mt;
        out[9] = P.mu;
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle_plan_stats: %s\n", e.what());
        return -1;
    }
}

// Host PSWF and quadrature of the product (checked against golden vectors).
int oracle_pswf(double beta, int nx, const double* x, double* psi, double* moments4) {
    pdmkb::Pswf0 pf(beta);
    for (int i = 0; i < nx; ++i) psi[i] = pf(x[i]);
    pf.moments(moments4[0], moments4[1], moments4[2], moments4[3]);
    return 0;
}

int oracle_legendre(int n, double* x, double* w) {
    pdmkb::gauss_legendre(n, x, w);
    return 0;
}

// Geometry of the host plan (for comparison with the reference's own image
// layout): returns the image count; fills umat, qmat, mgrid, xgrid0, rc and up
// to cap image source indices.
long oracle_plan_images(const double* cell, int n, const double* pos, int nz, double* umat, double* qmat, int* mgrid,
                        double* xgrid0, double* rc, int* img_idx, long cap) {
    try {
        Plan P = pdmkb::build_plan(cell, n, pos, 6, 1 << 30, nz);
        for (int i = 0; i < 9; ++i) {
            umat[i] = P.umat[i];
            qmat[i] = P.qmat[i];
        }
        for (int d = 0; d < 3; ++d) {
            mgrid[d] = P.mgrid[d];
            xgrid0[d] = P.xgrid0[d];
        }
        *rc = P.rc;
        for (long i = 0; i < (long)P.img_src_idx.size() && i < cap; ++i) img_idx[i] = P.img_src_idx[i];
        return (long)P.img_src_idx.size();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle_plan_images: %s\n", e.what());
        return -1;
    }
}

// Direct Ewald sum (neutral-gauge potentials, k = 0 dropped).  cell[j*3+i] =
// component i of lattice vector j; pos[3*i+d].  s sets the accuracy
// (erfc(s), exp(-s^2)).  energy = 1/2 sum q phi - pi Q^2 / (2 V alpha^2).
int oracle_ewald_direct(const double* cell, int n, const double* pos, const double* q, double s, double* pot,
                        double* energy) {
    const double* a0 = cell;
    const double* a1 = cell + 3;
    const double* a2 = cell + 6;
    auto cross = [](const double* u, const double* v, double* w) {
        w[0] = u[1] * v[2] - u[2] * v[1];
        w[1] = u[2] * v[0] - u[0] * v[2];
        w[2] = u[0] * v[1] - u[1] * v[0];
    };
    auto dot = [](const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
    double c12[3], c20[3], c01[3];
    cross(a1, a2, c12);
    cross(a2, a0, c20);
    cross(a0, a1, c01);
    const double V = std::fabs(dot(a0, c12));
    if (V <= 0) return -1;
    const double alpha = std::pow(n * M_PI * M_PI * M_PI / (V * V), 1.0 / 6.0);
    const double rcut = s / alpha, kmax = 2.0 * s * alpha;
    const double h[3] = {V / std::sqrt(dot(c12, c12)), V / std::sqrt(dot(c20, c20)), V / std::sqrt(dot(c01, c01))};
    int nmax[3];
    for (int d = 0; d < 3; ++d) nmax[d] = (int)std::ceil(rcut / h[d]);
    // reciprocal vectors b_d = 2 pi (a_{d+1} x a_{d+2}) / V
    double b[3][3];
    for (int d = 0; d < 3; ++d) {
        b[0][d] = 2 * M_PI * c12[d] / V;
        b[1][d] = 2 * M_PI * c20[d] / V;
        b[2][d] = 2 * M_PI * c01[d] / V;
    }
    // reciprocal-lattice heights: 2 pi / |a_d| along b_d directions
    int mmax[3];
    for (int d = 0; d < 3; ++d) {
        const double* ad = cell + 3 * d;
        mmax[d] = (int)std::ceil(kmax * std::sqrt(dot(ad, ad)) / (2 * M_PI));
    }
    std::vector<double> phi(n, 0.0);
    const double rc2 = rcut * rcut;
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < n; ++i) {
        double acc = 0;
        for (int j = 0; j < n; ++j)
            for (int n0 = -nmax[0]; n0 <= nmax[0]; ++n0)
                for (int n1 = -nmax[1]; n1 <= nmax[1]; ++n1)
                    for (int n2 = -nmax[2]; n2 <= nmax[2]; ++n2) {
                        if (i == j && n0 == 0 && n1 == 0 && n2 == 0) continue;
                        double dr[3];
                        for (int d = 0; d < 3; ++d)
                            dr[d] = pos[3 * i + d] - pos[3 * j + d] + n0 * a0[d] + n1 * a1[d] + n2 * a2[d];
                        const double r2 = dot(dr, dr);
                        if (r2 > rc2) continue;
                        const double r = std::sqrt(r2);
                        acc += q[j] * std::erfc(alpha * r) / r;
                    }
        phi[i] = acc;
    }
    const double km2 = kmax * kmax, inv4a2 = 1.0 / (4 * alpha * alpha), pref = 4 * M_PI / V;
    std::vector<std::array<double, 4>> ks;
    for (int m3 = -mmax[2]; m3 <= mmax[2]; ++m3)
        for (int m2 = -mmax[1]; m2 <= mmax[1]; ++m2)
            for (int m1 = -mmax[0]; m1 <= mmax[0]; ++m1) {
                if (!m1 && !m2 && !m3) continue;
                double kv[3];
                for (int d = 0; d < 3; ++d) kv[d] = m1 * b[0][d] + m2 * b[1][d] + m3 * b[2][d];
                const double k2 = dot(kv, kv);
                if (k2 > km2) continue;
                ks.push_back({kv[0], kv[1], kv[2], pref * std::exp(-k2 * inv4a2) / k2});
            }
    const int nk = (int)ks.size();
    std::vector<cplx> S(nk);
#pragma omp parallel for schedule(static)
    for (int m = 0; m < nk; ++m) {
        cplx s(0);
        for (int j = 0; j < n; ++j) {
            const double ph = ks[m][0] * pos[3 * j] + ks[m][1] * pos[3 * j + 1] + ks[m][2] * pos[3 * j + 2];
            s += q[j] * cplx(std::cos(ph), -std::sin(ph));
        }
        S[m] = s * ks[m][3];
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double acc = 0;
        for (int m = 0; m < nk; ++m) {
            const double ph = ks[m][0] * pos[3 * i] + ks[m][1] * pos[3 * i + 1] + ks[m][2] * pos[3 * i + 2];
            acc += S[m].real() * std::cos(ph) - S[m].imag() * std::sin(ph);
        }
        phi[i] += acc - 2.0 * alpha / std::sqrt(M_PI) * q[i];
    }
    double E = 0, Q = 0;
    for (int i = 0; i < n; ++i) {
        pot[i] = phi[i];
        E += q[i] * phi[i];
        Q += q[i];
    }
    if (energy) *energy = 0.5 * E - M_PI * Q * Q / (2 * V * alpha * alpha);
    return 0;
}

// Ewald sum at a subset of targets (neutral-gauge potentials, k = 0 dropped),
// for checks at sizes where the all-pairs sum above cannot finish:
//   phi(x_t) = sum_{j,n}' q_j erfc(alpha r)/r            (r = |x_t - x_j + R_n| < s/alpha)
//            + sum_{0 < |k| <= 2 s alpha} (4 pi / V) e^{-k^2/(4 alpha^2)} / k^2 Re[S(k) e^{i k.x_t}]
//            - 2 alpha/sqrt(pi) q_t,          S(k) = sum_j q_j e^{-i k.x_j}
// (the splitting of cpp/src/ewald_nufft.cpp:777-910, evaluated at m targets).
// Real space: sources binned in fractional coordinates; a pair closer than
// rcut differs by less than rcut/h_d in fractional coordinate d (h_d the
// lattice-plane spacing), which bounds the bins visited.  Reciprocal space:
// k.x = 2 pi (m . f) with f the fractional coordinates, so e^{-i k.x}
// factorises over the three axes and S(k) is accumulated per source over the
// modes of the sphere.  alpha <= 0 picks alpha from an estimate of the two
// costs.  Sums are compensated (Neumaier) so rounding stays near 1e-15 of the
// potential at 10^6 sources.
int oracle_ewald_targets_grad(const double* cell, int n, const double* pos, const double* q, int m, const int* tidx,
                              double s, double alpha, double* pot, double* grad);

int oracle_ewald_targets(const double* cell, int n, const double* pos, const double* q, int m, const int* tidx,
                         double s, double alpha, double* pot) {
    return oracle_ewald_targets_grad(cell, n, pos, q, m, tidx, s, alpha, pot, nullptr);
}

// The same with the potential's gradient at the targets: grad[3 ti + d] =
// d phi / d x_d (Cartesian; the field is -grad, the force on q_t is -q_t grad).
// Real space: d/dr [erfc(alpha r)/r] = -erfc(alpha r)/r^2 - 2 alpha/sqrt(pi) e^{-alpha^2 r^2}/r
// along (x_t - x_j)/r; reciprocal space: -sum w(k) k Im[S(k) e^{i k.x_t}].
int oracle_ewald_targets_grad(const double* cell, int n, const double* pos, const double* q, int m, const int* tidx,
                              double s, double alpha, double* pot, double* grad) {
    try {
        const double* a[3] = {cell, cell + 3, cell + 6};
        auto cross = [](const double* u, const double* v, double* w) {
            w[0] = u[1] * v[2] - u[2] * v[1];
            w[1] = u[2] * v[0] - u[0] * v[2];
            w[2] = u[0] * v[1] - u[1] * v[0];
        };
        auto dot = [](const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
        double c[3][3];
        cross(a[1], a[2], c[0]);
        cross(a[2], a[0], c[1]);
        cross(a[0], a[1], c[2]);
        const double V = std::fabs(dot(a[0], c[0]));
        if (!(V > 0) || n <= 0 || m <= 0) return -1;
        double h[3];
        for (int d = 0; d < 3; ++d) h[d] = V / std::sqrt(dot(c[d], c[d]));
        // fractional coordinates f = A^-1 x: rows of A^-1 are c_d / V (sign of det folded in)
        const double sgn = dot(a[0], c[0]) > 0 ? 1.0 : -1.0;
        double ainv[3][3];
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 3; ++e) ainv[d][e] = sgn * c[d][e] / V;
        if (!(alpha > 0)) {
            // real-space pairs ~ m * (n/V) * (4/3) pi rcut^3 * 10 (erfc, bins), reciprocal
            // modes ~ n * (4/3) pi kmax^3 V / (2 pi)^3
            const double A = m * (n / V) * 4.18879 * s * s * s * 10.0;
            const double B = n * 4.18879 * 8.0 * s * s * s * V / (8.0 * M_PI * M_PI * M_PI);
            alpha = std::pow(A / B, 1.0 / 6.0);
        }
        const double rcut = s / alpha, kmax = 2.0 * s * alpha, rc2 = rcut * rcut;
        std::vector<double> f((size_t)3 * n);
        for (int j = 0; j < n; ++j)
            for (int d = 0; d < 3; ++d) {
                const double* x = pos + 3 * (size_t)j;
                double v = ainv[d][0] * x[0] + ainv[d][1] * x[1] + ainv[d][2] * x[2];
                v -= std::floor(v);
                if (v >= 1.0) v = 0.0;
                f[3 * (size_t)j + d] = v;
            }
        // ---- real space
        int G[3], reach[3];
        const double per_bin = 8.0;  // target sources per bin
        const double nb = std::max(1.0, std::cbrt(n / per_bin));
        for (int d = 0; d < 3; ++d) {
            G[d] = std::max(1, std::min(512, (int)std::lround(nb)));
            reach[d] = (int)std::ceil(rcut / h[d] * G[d]) + 1;
        }
        const size_t nbins = (size_t)G[0] * G[1] * G[2];
        std::vector<int> bstart(nbins + 1, 0), border(n);
        auto bin_of = [&](int j) {
            int b[3];
            for (int d = 0; d < 3; ++d) b[d] = std::min(G[d] - 1, (int)(f[3 * (size_t)j + d] * G[d]));
            return ((size_t)b[2] * G[1] + b[1]) * G[0] + b[0];
        };
        for (int j = 0; j < n; ++j) bstart[bin_of(j) + 1]++;
        for (size_t b = 0; b < nbins; ++b) bstart[b + 1] += bstart[b];
        {
            std::vector<int> fill(bstart.begin(), bstart.end() - 1);
            for (int j = 0; j < n; ++j) border[fill[bin_of(j)]++] = j;
        }
        std::vector<double> phi(m, 0.0), gr((size_t)3 * m, 0.0);
        const double twoa_sqpi = 2.0 * alpha / std::sqrt(M_PI);
#pragma omp parallel for schedule(dynamic, 1)
        for (int ti = 0; ti < m; ++ti) {
            const int t = tidx[ti];
            const double* ft = &f[3 * (size_t)t];
            int bt[3];
            for (int d = 0; d < 3; ++d) bt[d] = std::min(G[d] - 1, (int)(ft[d] * G[d]));
            double sum = 0, comp = 0, g0 = 0, g1 = 0, g2 = 0;
            for (int o2 = -reach[2]; o2 <= reach[2]; ++o2)
                for (int o1 = -reach[1]; o1 <= reach[1]; ++o1)
                    for (int o0 = -reach[0]; o0 <= reach[0]; ++o0) {
                        const int raw[3] = {bt[0] + o0, bt[1] + o1, bt[2] + o2};
                        int bi[3], sh[3];
                        for (int d = 0; d < 3; ++d) {
                            sh[d] = (int)std::floor((double)raw[d] / G[d]);
                            bi[d] = raw[d] - sh[d] * G[d];
                        }
                        const size_t b = ((size_t)bi[2] * G[1] + bi[1]) * G[0] + bi[0];
                        for (int k = bstart[b]; k < bstart[b + 1]; ++k) {
                            const int j = border[k];
                            if (j == t && !sh[0] && !sh[1] && !sh[2]) continue;
                            double df[3];
                            for (int d = 0; d < 3; ++d) df[d] = ft[d] - (f[3 * (size_t)j + d] + sh[d]);
                            double dr[3];
                            for (int e = 0; e < 3; ++e) dr[e] = a[0][e] * df[0] + a[1][e] * df[1] + a[2][e] * df[2];
                            const double r2 = dot(dr, dr);
                            if (r2 >= rc2) continue;
                            const double r = std::sqrt(r2);
                            const double ec = std::erfc(alpha * r);
                            const double v = q[j] * ec / r;
                            const double tsum = sum + v;
                            comp += std::fabs(sum) >= std::fabs(v) ? (sum - tsum) + v : (v - tsum) + sum;
                            sum = tsum;
                            if (grad) {
                                const double dvdr = -q[j] * (ec / r2 + twoa_sqpi * std::exp(-alpha * alpha * r2) / r);
                                g0 += dvdr * dr[0] / r;
                                g1 += dvdr * dr[1] / r;
                                g2 += dvdr * dr[2] / r;
                            }
                        }
                    }
            phi[ti] = sum + comp - 2.0 * alpha / std::sqrt(M_PI) * q[t];
            gr[3 * (size_t)ti] = g0;
            gr[3 * (size_t)ti + 1] = g1;
            gr[3 * (size_t)ti + 2] = g2;
        }
        // ---- reciprocal space: modes m with |m1 b1 + m2 b2 + m3 b3| <= kmax
        double b[3][3];
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 3; ++e) b[d][e] = 2 * M_PI * ainv[d][e];
        int mm[3];
        for (int d = 0; d < 3; ++d) mm[d] = (int)std::ceil(kmax * std::sqrt(dot(a[d], a[d])) / (2 * M_PI));
        struct Row {
            int m2, m3, lo, hi;  // m1 in [lo, hi]
            size_t off;
        };
        std::vector<Row> rows;
        std::vector<double> w;
        const double km2 = kmax * kmax, inv4a2 = 1.0 / (4 * alpha * alpha), pref = 4 * M_PI / V;
        size_t nk = 0;
        for (int m3 = 0; m3 <= mm[2]; ++m3)
            for (int m2 = -mm[1]; m2 <= mm[1]; ++m2) {
                if (m3 == 0 && m2 < 0) continue;  // half space: (m3 > 0) or (m3 = 0, m2 > 0) or (m3 = m2 = 0, m1 > 0)
                int lo = -mm[0], hi = mm[0];
                if (m3 == 0 && m2 == 0) lo = 1;
                Row r{m2, m3, 0, -1, nk};
                for (int m1 = lo; m1 <= hi; ++m1) {
                    double kv[3];
                    for (int e = 0; e < 3; ++e) kv[e] = m1 * b[0][e] + m2 * b[1][e] + m3 * b[2][e];
                    const double k2 = dot(kv, kv);
                    if (k2 > km2) continue;
                    if (r.hi < r.lo) r.lo = m1;
                    r.hi = m1;
                }
                if (r.hi < r.lo) continue;
                for (int m1 = r.lo; m1 <= r.hi; ++m1) {
                    double kv[3];
                    for (int e = 0; e < 3; ++e) kv[e] = m1 * b[0][e] + m2 * b[1][e] + m3 * b[2][e];
                    const double k2 = dot(kv, kv);
                    w.push_back(k2 <= km2 ? 2.0 * pref * std::exp(-k2 * inv4a2) / k2 : 0.0);  // x2: the -k half
                }
                nk += r.hi - r.lo + 1;
                rows.push_back(r);
            }
        std::vector<cplx> S(nk, cplx(0));
        const int nthreads = omp_get_max_threads();
        const int chunk = 512;
#pragma omp parallel num_threads(nthreads)
        {
            std::vector<cplx> acc(nk, cplx(0)), part(nk, cplx(0));
            std::vector<cplx> e1(2 * mm[0] + 1), e2(2 * mm[1] + 1), e3(mm[2] + 1);
#pragma omp for schedule(static)
            for (int c0 = 0; c0 < n; c0 += chunk) {
                std::fill(part.begin(), part.end(), cplx(0));
                for (int j = c0; j < std::min(n, c0 + chunk); ++j) {
                    const double* fj = &f[3 * (size_t)j];
                    for (int k = -mm[0]; k <= mm[0]; ++k)
                        e1[k + mm[0]] = std::polar(1.0, -2 * M_PI * k * fj[0]);
                    for (int k = -mm[1]; k <= mm[1]; ++k)
                        e2[k + mm[1]] = std::polar(1.0, -2 * M_PI * k * fj[1]);
                    for (int k = 0; k <= mm[2]; ++k) e3[k] = std::polar(1.0, -2 * M_PI * k * fj[2]);
                    for (const Row& r : rows) {
                        const cplx g = q[j] * e3[r.m3] * e2[r.m2 + mm[1]];
                        cplx* pp = &part[r.off];
                        const cplx* ee = &e1[r.lo + mm[0]];
                        for (int k = 0; k <= r.hi - r.lo; ++k) pp[k] += g * ee[k];
                    }
                }
                for (size_t k = 0; k < nk; ++k) acc[k] += part[k];
            }
#pragma omp critical
            for (size_t k = 0; k < nk; ++k) S[k] += acc[k];
        }
#pragma omp parallel for schedule(dynamic, 1)
        for (int ti = 0; ti < m; ++ti) {
            const double* ft = &f[3 * (size_t)tidx[ti]];
            std::vector<cplx> e1(2 * mm[0] + 1), e2(2 * mm[1] + 1), e3(mm[2] + 1);
            for (int k = -mm[0]; k <= mm[0]; ++k) e1[k + mm[0]] = std::polar(1.0, 2 * M_PI * k * ft[0]);
            for (int k = -mm[1]; k <= mm[1]; ++k) e2[k + mm[1]] = std::polar(1.0, 2 * M_PI * k * ft[1]);
            for (int k = 0; k <= mm[2]; ++k) e3[k] = std::polar(1.0, 2 * M_PI * k * ft[2]);
            double sum = 0, comp = 0, g0 = 0, g1 = 0, g2 = 0;
            for (const Row& r : rows) {
                const cplx g = e3[r.m3] * e2[r.m2 + mm[1]];
                for (int k = 0; k <= r.hi - r.lo; ++k) {
                    const cplx zv = S[r.off + k] * g * e1[r.lo + k + mm[0]];
                    const double v = w[r.off + k] * zv.real();
                    const double tsum = sum + v;
                    comp += std::fabs(sum) >= std::fabs(v) ? (sum - tsum) + v : (v - tsum) + sum;
                    sum = tsum;
                    if (grad) {
                        const int m1 = r.lo + k;
                        const double wi = -w[r.off + k] * zv.imag();
                        g0 += wi * (m1 * b[0][0] + r.m2 * b[1][0] + r.m3 * b[2][0]);
                        g1 += wi * (m1 * b[0][1] + r.m2 * b[1][1] + r.m3 * b[2][1]);
                        g2 += wi * (m1 * b[0][2] + r.m2 * b[1][2] + r.m3 * b[2][2]);
                    }
                }
            }
            pot[ti] = phi[ti] + sum + comp;
            if (grad) {
                grad[3 * (size_t)ti] = gr[3 * (size_t)ti] + g0;
                grad[3 * (size_t)ti + 1] = gr[3 * (size_t)ti + 1] + g1;
                grad[3 * (size_t)ti + 2] = gr[3 * (size_t)ti + 2] + g2;
            }
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle_ewald_targets: %s\n", e.what());
        return -1;
    }
}

// k charge vectors on one plan (charges and potentials N x k column-major);
// the exact far field, as oracle_evaluate.
int oracle_evaluate_multi(const double* cell, int n, const double* pos, int k, const double* Q, int n_digits,
                          int n_per_leaf, int nz, double* pot) {
    try {
        Plan P = pdmkb::build_plan(cell, n, pos, n_digits, n_per_leaf, nz);
        for (int c = 0; c < k; ++c) {
            Components C;
            oracle_eval(P, Q + (size_t)n * c, C, true, false);
            double* out = pot + (size_t)n * c;
            for (int i = 0; i < n; ++i) out[i] = C.near[i] + C.mid[i] + C.self[i] + C.far[i];
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle_evaluate_multi: %s\n", e.what());
        return -1;
    }
}

// Quasi-periodic Ewald sum at a subset of targets: images at x_j + R carry the
// phase e^{i beta.R} (beta the Bloch vector, Cartesian, the caller's frame):
//   phi(x_t) = sum_{j,R}' q_j e^{i beta.R} G(x_t - x_j - R), G = 1/r,
// split as erfc(alpha r)/r (real space, R = (x_t - x_j) - dr from the actual
// positions) + the Bloch-periodised erf(alpha r)/r,
//   (4 pi / V) sum_k e^{-|k+beta|^2/(4 alpha^2)} / |k+beta|^2 S(k) e^{i (k+beta).x_t},
//   S(k) = sum_j q_j e^{-i (k+beta).x_j}   (all k; k + beta = 0 dropped)
// - 2 alpha/sqrt(pi) q_t.  The periodic sum is the beta = 0 case.  Complex
// output (pot_re, pot_im).
int oracle_ewald_targets_qp(const double* cell, int n, const double* pos, const double* q, int m, const int* tidx,
                            double s, double alpha, const double* bloch, double* pot_re, double* pot_im) {
    try {
        const double* a[3] = {cell, cell + 3, cell + 6};
        auto cross = [](const double* u, const double* v, double* w) {
            w[0] = u[1] * v[2] - u[2] * v[1];
            w[1] = u[2] * v[0] - u[0] * v[2];
            w[2] = u[0] * v[1] - u[1] * v[0];
        };
        auto dot = [](const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
        double c[3][3];
        cross(a[1], a[2], c[0]);
        cross(a[2], a[0], c[1]);
        cross(a[0], a[1], c[2]);
        const double V = std::fabs(dot(a[0], c[0]));
        if (!(V > 0) || n <= 0 || m <= 0) return -1;
        double h[3];
        for (int d = 0; d < 3; ++d) h[d] = V / std::sqrt(dot(c[d], c[d]));
        const double sgn = dot(a[0], c[0]) > 0 ? 1.0 : -1.0;
        double ainv[3][3];
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 3; ++e) ainv[d][e] = sgn * c[d][e] / V;
        if (!(alpha > 0)) {
            const double A = m * (n / V) * 4.18879 * s * s * s * 10.0;
            const double B = 2.0 * n * 4.18879 * 8.0 * s * s * s * V / (8.0 * M_PI * M_PI * M_PI);
            alpha = std::pow(A / B, 1.0 / 6.0);
        }
        const double rcut = s / alpha, kmax = 2.0 * s * alpha, rc2 = rcut * rcut;
        std::vector<double> f((size_t)3 * n), fu((size_t)3 * n);
        for (int j = 0; j < n; ++j)
            for (int d = 0; d < 3; ++d) {
                const double* x = pos + 3 * (size_t)j;
                const double v = ainv[d][0] * x[0] + ainv[d][1] * x[1] + ainv[d][2] * x[2];
                fu[3 * (size_t)j + d] = v;
                double w = v - std::floor(v);
                if (w >= 1.0) w = 0.0;
                f[3 * (size_t)j + d] = w;
            }
        // ---- real space (cell list as oracle_ewald_targets)
        int G[3], reach[3];
        const double nb = std::max(1.0, std::cbrt(n / 8.0));
        for (int d = 0; d < 3; ++d) {
            G[d] = std::max(1, std::min(512, (int)std::lround(nb)));
            reach[d] = (int)std::ceil(rcut / h[d] * G[d]) + 1;
        }
        const size_t nbins = (size_t)G[0] * G[1] * G[2];
        std::vector<int> bstart(nbins + 1, 0), border(n);
        auto bin_of = [&](int j) {
            int b[3];
            for (int d = 0; d < 3; ++d) b[d] = std::min(G[d] - 1, (int)(f[3 * (size_t)j + d] * G[d]));
            return ((size_t)b[2] * G[1] + b[1]) * G[0] + b[0];
        };
        for (int j = 0; j < n; ++j) bstart[bin_of(j) + 1]++;
        for (size_t b = 0; b < nbins; ++b) bstart[b + 1] += bstart[b];
        {
            std::vector<int> fill(bstart.begin(), bstart.end() - 1);
            for (int j = 0; j < n; ++j) border[fill[bin_of(j)]++] = j;
        }
        std::vector<cplx> phi(m);
#pragma omp parallel for schedule(dynamic, 1)
        for (int ti = 0; ti < m; ++ti) {
            const int t = tidx[ti];
            const double* ft = &f[3 * (size_t)t];
            const double* xt = pos + 3 * (size_t)t;
            int bt[3];
            for (int d = 0; d < 3; ++d) bt[d] = std::min(G[d] - 1, (int)(ft[d] * G[d]));
            cplx sum(0);
            for (int o2 = -reach[2]; o2 <= reach[2]; ++o2)
                for (int o1 = -reach[1]; o1 <= reach[1]; ++o1)
                    for (int o0 = -reach[0]; o0 <= reach[0]; ++o0) {
                        const int raw[3] = {bt[0] + o0, bt[1] + o1, bt[2] + o2};
                        int bi[3], sh[3];
                        for (int d = 0; d < 3; ++d) {
                            sh[d] = (int)std::floor((double)raw[d] / G[d]);
                            bi[d] = raw[d] - sh[d] * G[d];
                        }
                        const size_t b = ((size_t)bi[2] * G[1] + bi[1]) * G[0] + bi[0];
                        for (int k = bstart[b]; k < bstart[b + 1]; ++k) {
                            const int j = border[k];
                            if (j == t && !sh[0] && !sh[1] && !sh[2]) continue;
                            double df[3];
                            for (int d = 0; d < 3; ++d) df[d] = ft[d] - (f[3 * (size_t)j + d] + sh[d]);
                            double dr[3];
                            for (int e = 0; e < 3; ++e) dr[e] = a[0][e] * df[0] + a[1][e] * df[1] + a[2][e] * df[2];
                            const double r2 = dot(dr, dr);
                            if (r2 >= rc2) continue;
                            const double r = std::sqrt(r2);
                            const double* xj = pos + 3 * (size_t)j;
                            double R[3];
                            for (int e = 0; e < 3; ++e) R[e] = (xt[e] - xj[e]) - dr[e];
                            const double ph = dot(bloch, R);
                            sum += q[j] * std::erfc(alpha * r) / r * cplx(std::cos(ph), std::sin(ph));
                        }
                    }
            phi[ti] = sum - 2.0 * alpha / std::sqrt(M_PI) * q[t];
        }
        // ---- reciprocal space: every mode m with |2 pi A^-T m + beta| <= kmax
        double b[3][3];
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 3; ++e) b[d][e] = 2 * M_PI * ainv[d][e];
        const double bn = std::sqrt(dot(bloch, bloch));
        int mm[3];
        for (int d = 0; d < 3; ++d) mm[d] = (int)std::ceil((kmax + bn) * std::sqrt(dot(a[d], a[d])) / (2 * M_PI));
        std::vector<std::array<int, 3>> modes;
        std::vector<double> w;
        const double km2 = kmax * kmax, inv4a2 = 1.0 / (4 * alpha * alpha), pref = 4 * M_PI / V;
        for (int m3 = -mm[2]; m3 <= mm[2]; ++m3)
            for (int m2 = -mm[1]; m2 <= mm[1]; ++m2)
                for (int m1 = -mm[0]; m1 <= mm[0]; ++m1) {
                    double kv[3];
                    for (int e = 0; e < 3; ++e) kv[e] = m1 * b[0][e] + m2 * b[1][e] + m3 * b[2][e] + bloch[e];
                    const double k2 = dot(kv, kv);
                    if (k2 > km2 || k2 < 1e-24) continue;
                    modes.push_back({m1, m2, m3});
                    w.push_back(pref * std::exp(-k2 * inv4a2) / k2);
                }
        const size_t nk = modes.size();
        std::vector<cplx> S(nk, cplx(0));
#pragma omp parallel
        {
            std::vector<cplx> acc(nk, cplx(0));
            std::vector<cplx> e1(2 * mm[0] + 1), e2(2 * mm[1] + 1), e3(2 * mm[2] + 1);
#pragma omp for schedule(static)
            for (int j = 0; j < n; ++j) {
                const double* fj = &fu[3 * (size_t)j];
                const double bx = dot(bloch, pos + 3 * (size_t)j);
                const cplx cj = q[j] * cplx(std::cos(bx), -std::sin(bx));
                for (int k = -mm[0]; k <= mm[0]; ++k) e1[k + mm[0]] = std::polar(1.0, -2 * M_PI * k * fj[0]);
                for (int k = -mm[1]; k <= mm[1]; ++k) e2[k + mm[1]] = std::polar(1.0, -2 * M_PI * k * fj[1]);
                for (int k = -mm[2]; k <= mm[2]; ++k) e3[k + mm[2]] = std::polar(1.0, -2 * M_PI * k * fj[2]);
                for (size_t k = 0; k < nk; ++k)
                    acc[k] += cj * e1[modes[k][0] + mm[0]] * e2[modes[k][1] + mm[1]] * e3[modes[k][2] + mm[2]];
            }
#pragma omp critical
            for (size_t k = 0; k < nk; ++k) S[k] += acc[k];
        }
#pragma omp parallel for schedule(dynamic, 1)
        for (int ti = 0; ti < m; ++ti) {
            const int t = tidx[ti];
            const double* ft = &fu[3 * (size_t)t];
            cplx sum(0);
            for (size_t k = 0; k < nk; ++k) {
                const double ph = 2 * M_PI * (modes[k][0] * ft[0] + modes[k][1] * ft[1] + modes[k][2] * ft[2]);
                sum += w[k] * S[k] * cplx(std::cos(ph), std::sin(ph));
            }
            const double bx = dot(bloch, pos + 3 * (size_t)t);
            const cplx v = phi[ti] + sum * cplx(std::cos(bx), std::sin(bx));
            pot_re[ti] = v.real();
            pot_im[ti] = v.imag();
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle_ewald_targets_qp: %s\n", e.what());
        return -1;
    }
}

}  // extern "C"
