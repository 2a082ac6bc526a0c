// Geometry, lattice images and the adaptive tree for one periodic system.
//
// The construction rules reproduce the reference exactly, so that the boxes,
// leaf populations and interaction lists (and therefore the potentials) match:
//   lattice_setup / compute_grid   cpp/include/dmk/pbc.hpp:23-117
//   images (+ source index)        cpp/include/pdmk/image_layout.hpp:14-88
//   level-0 grid + bin sort        cpp/include/dmk/pbc.hpp:265-391
//   refinement, colleagues         cpp/src/dmk/pbc_tree.cpp:306-428
//   2:1 balance                    cpp/src/dmk/pbc_tree.cpp:438-598
//   flags, lists, work lists       cpp/src/dmk/pbc_tree.cpp:776-1011
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <stdexcept>

#include "plan.hpp"
#include "points.hpp"

namespace pdmkb {

void build_tables(Plan& P);  // tables.cpp

namespace {

// QR of the lattice with columns ordered by decreasing length
// (cpp/include/dmk/pbc.hpp:23-101); umat upper triangular.
void lattice_setup(const double* avec, double* umat, double* qmat) {
    double anorm[3];
    int iord[3];
    for (int i = 0; i < 3; i++) {
        double s = 0;
        for (int k = 0; k < 3; k++) s += avec[k + i * 3] * avec[k + i * 3];
        anorm[i] = std::sqrt(s);
        iord[i] = i;
    }
    for (int i = 0; i < 2; i++)
        for (int j = i + 1; j < 3; j++)
            if (anorm[j] > anorm[i]) {
                std::swap(anorm[i], anorm[j]);
                std::swap(iord[i], iord[j]);
            }
    double as[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) as[j + i * 3] = avec[j + iord[i] * 3];
    // Modified Gram-Schmidt, column by column.
    const double r11 = anorm[0];
    for (int i = 0; i < 3; i++) qmat[i] = as[i] / r11;
    double r12 = 0;
    for (int i = 0; i < 3; i++) r12 += qmat[i] * as[i + 3];
    for (int i = 0; i < 3; i++) qmat[i + 3] = as[i + 3] - r12 * qmat[i];
    double r22 = 0;
    for (int i = 0; i < 3; i++) r22 += qmat[i + 3] * qmat[i + 3];
    r22 = std::sqrt(r22);
    for (int i = 0; i < 3; i++) qmat[i + 3] /= r22;
    double r13 = 0, r23 = 0, r33 = 0;
    for (int i = 0; i < 3; i++) {
        r13 += qmat[i] * as[i + 6];
        r23 += qmat[i + 3] * as[i + 6];
    }
    for (int i = 0; i < 3; i++) qmat[i + 6] = as[i + 6] - r13 * qmat[i] - r23 * qmat[i + 3];
    for (int i = 0; i < 3; i++) r33 += qmat[i + 6] * qmat[i + 6];
    r33 = std::sqrt(r33);
    for (int i = 0; i < 3; i++) qmat[i + 6] /= r33;
    for (int i = 0; i < 9; i++) umat[i] = 0;
    umat[0] = r11;
    umat[3] = r12;
    umat[4] = r22;
    umat[6] = r13;
    umat[7] = r23;
    umat[8] = r33;
}

void compute_grid(const double* umat, double rc, int* mgrid, double* xgrid0) {
    for (int i = 2; i >= 0; i--) {
        double xmin = 0, xmax = umat[i + i * 3];
        for (int j = i + 1; j < 3; j++) {
            const double v = umat[i + j * 3];
            xmin += std::min(0.0, v);
            xmax += std::max(0.0, v);
        }
        mgrid[i] = std::max(1, (int)std::ceil((xmax - xmin) / rc));
        xgrid0[i] = xmin;
    }
}

void utri_inv(const double* u, double* v) {
    for (int i = 0; i < 9; i++) v[i] = 0;
    v[0] = 1.0 / u[0];
    v[4] = 1.0 / u[4];
    v[3] = -u[3] / (u[0] * u[4]);
    v[8] = 1.0 / u[8];
    v[7] = -u[7] / (u[4] * u[8]);
    v[6] = (u[3] * u[7] - u[6] * u[4]) / (u[0] * u[4] * u[8]);
}

// Lattice images of the originals that fall in the extended grid (one rc
// layer around the inner grid).  The shift loop order is the reference's, so
// the image list, and hence the sort, is identical: image_shifts lists the
// candidate shifts in that order, and for each shift every original whose
// shifted copy lies in [lo_ext, hi_ext] is appended in input order.
void image_shifts(const double* umat, double rc, const int* mgrid, const double* xgrid0,
                  std::vector<std::array<double, 3>>& shifts, double* lo_ext, double* hi_ext) {
    double lo[3], hi[3];
    for (int i = 0; i < 3; ++i) {
        lo_ext[i] = xgrid0[i] - rc;
        hi_ext[i] = xgrid0[i] + (mgrid[i] + 1) * rc;
        lo[i] = xgrid0[i];
        double w = umat[i + i * 3];
        for (int j = i + 1; j < 3; ++j) w += std::abs(umat[i + j * 3]);
        hi[i] = xgrid0[i] + w;
    }
    shifts.clear();
    const int n3max = (int)((mgrid[2] + 1) * rc / umat[8]) + 1;
    for (int n3 = -n3max; n3 <= n3max; ++n3) {
        const double s3 = umat[8] * n3;
        if (lo[2] + s3 > hi_ext[2] || hi[2] + s3 < lo_ext[2]) continue;
        const int n2max = (int)(((mgrid[1] + 1) * rc + std::abs(umat[7] * n3)) / umat[4]) + 1;
        for (int n2 = -n2max; n2 <= n2max; ++n2) {
            const double s2 = umat[4] * n2 + umat[7] * n3;
            if (lo[1] + s2 > hi_ext[1] || hi[1] + s2 < lo_ext[1]) continue;
            const double off = umat[3] * n2 + umat[6] * n3;
            const int n1max = (int)(((mgrid[0] + 1) * rc + std::abs(off)) / umat[0]) + 1;
            for (int n1 = -n1max; n1 <= n1max; ++n1) {
                if (n1 == 0 && n2 == 0 && n3 == 0) continue;
                const double s1 = umat[0] * n1 + off;
                if (lo[0] + s1 > hi_ext[0] || hi[0] + s1 < lo_ext[0]) continue;
                shifts.push_back({s1, s2, s3});
            }
        }
    }
}


uint64_t spread3(uint32_t v) {  // 10 bits -> every third bit of 30
    uint64_t x = v & 0x3FF;
    x = (x | (x << 16)) & 0x030000FF;
    x = (x | (x << 8)) & 0x0300F00F;
    x = (x | (x << 4)) & 0x030C30C3;
    x = (x | (x << 2)) & 0x09249249;
    return x;
}

// The point steps on the host.
class HostPoints final : public PointOps {
  public:
    void load(int n, const double* r) override {
        for (int s = 0; s < 2; ++s) {
            pos_[s].assign(r, r + 3 * (size_t)n);
            perm_[s].resize(n);
            for (int i = 0; i < n; ++i) perm_[s][i] = i;
        }
        n_ = n;
    }
    std::vector<int> add_images(const std::vector<std::array<double, 3>>& shifts, const double* lo,
                                const double* hi) override {
        std::vector<int> idx;
        std::vector<double>& x = pos_[0];
        for (const auto& sh : shifts)
            for (int j = 0; j < n_; ++j) {
                const double x0 = x[3 * (size_t)j] + sh[0], x1 = x[3 * (size_t)j + 1] + sh[1],
                             x2 = x[3 * (size_t)j + 2] + sh[2];
                if (x0 < lo[0] || x0 > hi[0] || x1 < lo[1] || x1 > hi[1] || x2 < lo[2] || x2 > hi[2]) continue;
                x.insert(x.end(), {x0, x1, x2});
                idx.push_back(j);
            }
        const int na = (int)(x.size() / 3);
        perm_[0].resize(na);
        for (int i = 0; i < na; ++i) perm_[0][i] = i;
        return idx;
    }
    std::vector<int> bin0(int s, const double* xelo, double rcinv, const int* m) override {
        const std::vector<double>& x = pos_[s];
        const int np = size(s), nb0 = m[0] * m[1] * m[2];
        std::vector<int> boxof(np), ip(nb0 + 1, 0);
        for (int i = 0; i < np; ++i) {
            int ii[3];
            for (int k = 0; k < 3; ++k) {
                ii[k] = (int)((x[3 * (size_t)i + k] - xelo[k]) * rcinv);
                ii[k] = std::min(std::max(ii[k], 0), m[k] - 1);
            }
            boxof[i] = ii[2] * m[0] * m[1] + ii[1] * m[0] + ii[0];
            ip[boxof[i] + 1]++;
        }
        for (int b = 0; b < nb0; ++b) ip[b + 1] += ip[b];
        std::vector<int> fill(ip.begin(), ip.end() - 1), perm(np);
        for (int i = 0; i < np; ++i) perm[fill[boxof[i]]++] = i;
        std::vector<double> sorted(3 * (size_t)np);
        std::vector<int> sp(np);
        for (int i = 0; i < np; ++i) {
            for (int d = 0; d < 3; ++d) sorted[3 * (size_t)i + d] = x[3 * (size_t)perm[i] + d];
            sp[i] = perm_[s][perm[i]];
        }
        pos_[s] = std::move(sorted);
        perm_[s] = std::move(sp);
        return ip;
    }
    std::vector<std::array<int, 8>> partition(int s, const std::vector<Range>& r) override {
        std::vector<std::array<int, 8>> out(r.size());
        std::vector<double>& pos = pos_[s];
        std::vector<int>& perm = perm_[s];
        for (size_t k = 0; k < r.size(); ++k) {
            const int start = r[k].start, npts = r[k].count;
            std::vector<int> oct(npts);
            std::array<int, 8> cnt{};
            for (int i = 0; i < npts; ++i) {
                int o = 0;
                for (int d = 0; d < 3; ++d)
                    if (pos[3 * (size_t)(start + i) + d] >= r[k].c[d]) o |= (1 << d);
                oct[i] = o;
                cnt[o]++;
            }
            int run[8];
            run[0] = start;
            for (int c = 1; c < 8; ++c) run[c] = run[c - 1] + cnt[c - 1];
            std::vector<double> tp(pos.begin() + 3 * (size_t)start, pos.begin() + 3 * (size_t)(start + npts));
            std::vector<int> tq(perm.begin() + start, perm.begin() + start + npts);
            for (int i = 0; i < npts; ++i) {
                const int g = run[oct[i]]++;
                for (int d = 0; d < 3; ++d) pos[3 * (size_t)g + d] = tp[3 * (size_t)i + d];
                perm[g] = tq[i];
            }
            out[k] = cnt;
        }
        return out;
    }
    void morton(int s, const std::vector<Leaf>& leaves) override {
        std::vector<double>& pos = pos_[s];
        std::vector<int>& perm = perm_[s];
        for (const Leaf& L : leaves) {
            const int start = L.start, count = L.count;
            if (count < 2) continue;
            std::vector<uint64_t> key(count);
            std::vector<int> order(count);
            for (int i = 0; i < count; ++i) {
                uint64_t k = 0;
                for (int d = 0; d < 3; ++d) {
                    const double f = (pos[3 * (size_t)(start + i) + d] - (L.c[d] - L.h)) / (2.0 * L.h);
                    const int qd = std::min(1023, std::max(0, (int)(f * 1024.0)));
                    k |= spread3((uint32_t)qd) << d;
                }
                key[i] = k;
                order[i] = i;
            }
            std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return key[a] < key[c]; });
            std::vector<double> tp(pos.begin() + 3 * (size_t)start, pos.begin() + 3 * (size_t)(start + count));
            std::vector<int> tq(perm.begin() + start, perm.begin() + start + count);
            for (int i = 0; i < count; ++i) {
                for (int d = 0; d < 3; ++d) pos[3 * (size_t)(start + i) + d] = tp[3 * (size_t)order[i] + d];
                perm[start + i] = tq[order[i]];
            }
        }
    }
    int64_t outside(int s, const std::vector<Leaf>& leaves) override {
        int64_t bad = 0;
        for (const Leaf& L : leaves)
            for (int i = L.start; i < L.start + L.count; ++i)
                for (int d = 0; d < 3; ++d)
                    if (std::abs(pos_[s][3 * (size_t)i + d] - L.c[d]) > L.h) {
                        ++bad;
                        break;
                    }
        return bad;
    }
    void fetch(int s, std::vector<double>& pos, std::vector<int>& perm) override {
        pos = pos_[s];
        perm = perm_[s];
    }
    int size(int s) const override { return (int)perm_[s].size(); }

  private:
    int n_ = 0;
    std::vector<double> pos_[2];
    std::vector<int> perm_[2];
};

inline int child_sign(int c, int d) { return ((c >> d) & 1) ? 1 : -1; }

// Working state of the builder: box topology grows as boxes split.
struct Builder {
    std::vector<int> depth, parent, nchild, ncoll;
    std::vector<std::array<int, 8>> children;
    std::vector<std::array<int, 27>> coll;
    std::vector<double> cen;  // 3 per box
    std::vector<int> sse, tse;  // [start, end] inclusive per box, end = start-1 if empty
    PointOps* ops = nullptr;    // where the points live
    std::vector<int> pending;   // split boxes whose points are not yet partitioned

    int add_box(int d, int par) {
        const int id = (int)depth.size();
        depth.push_back(d);
        parent.push_back(par);
        nchild.push_back(0);
        ncoll.push_back(0);
        children.push_back({});
        children.back().fill(-1);
        coll.push_back({});
        coll.back().fill(-1);
        cen.insert(cen.end(), {0.0, 0.0, 0.0});
        sse.insert(sse.end(), {0, -1});
        tse.insert(tse.end(), {0, -1});
        return id;
    }
    int nbox() const { return (int)depth.size(); }
    int scount(int b) const { return sse[2 * b + 1] - sse[2 * b] + 1; }
    int tcount(int b) const { return tse[2 * b + 1] - tse[2 * b] + 1; }

    // Create the 8 children of b (depth L -> L+1); their points are
    // distributed by the next flush.
    void split(int b, int L, double rc) {
        const double bsh = rc / (double)(1 << (L + 2));
        nchild[b] = 8;
        for (int c = 0; c < 8; ++c) {
            const int id = add_box(L + 1, b);
            children[b][c] = id;
            for (int d = 0; d < 3; ++d) cen[3 * id + d] = cen[3 * b + d] + child_sign(c, d) * bsh;
        }
        pending.push_back(b);
    }

    // Stable partition of every pending box's points into its children by the
    // octant relative to the box centre (>= means upper half).  The ranges of
    // different boxes are disjoint, so one batch gives the same result as
    // partitioning each box as it splits.
    void flush() {
        if (pending.empty()) return;
        for (int s = 0; s < 2; ++s) {
            std::vector<int>& se = s == 0 ? sse : tse;
            std::vector<PointOps::Range> r;
            std::vector<int> who;
            for (int b : pending) {
                const int cnt = se[2 * b + 1] - se[2 * b] + 1;
                if (cnt <= 0) continue;
                r.push_back({se[2 * b], cnt, {cen[3 * b], cen[3 * b + 1], cen[3 * b + 2]}});
                who.push_back(b);
            }
            if (r.empty()) continue;
            const std::vector<std::array<int, 8>> counts = ops->partition(s, r);
            for (size_t k = 0; k < who.size(); ++k) {
                int off = r[k].start;
                for (int c = 0; c < 8; ++c) {
                    const int ch = children[who[k]][c];
                    se[2 * ch] = off;
                    se[2 * ch + 1] = off + counts[k][c] - 1;
                    off += counts[k][c];
                }
            }
        }
        pending.clear();
    }

    // Colleague list of box nb (depth L+1) from the children of its parent's
    // non-leaf colleagues.
    void child_colleagues(int nb, double child_bs) {
        const int dad = parent[nb];
        const double tol = 1.05 * child_bs;
        ncoll[nb] = 0;
        coll[nb].fill(-1);
        for (int ic = 0; ic < 27; ++ic) {
            const int jb = coll[dad][ic];
            if (jb < 0 || nchild[jb] == 0) continue;
            for (int jc = 0; jc < 8; ++jc) {
                const int kb = children[jb][jc];
                if (kb < 0) continue;
                bool adj = true;
                for (int d = 0; d < 3; ++d)
                    if (std::abs(cen[3 * nb + d] - cen[3 * kb + d]) > tol) {
                        adj = false;
                        break;
                    }
                if (!adj) continue;
                int s = 0, st = 1;
                for (int d = 0; d < 3; ++d) {
                    const int di = (int)std::round((cen[3 * kb + d] - cen[3 * nb + d]) / child_bs);
                    s += (di + 1) * st;
                    st *= 3;
                }
                if (s >= 0 && s < 27) {
                    coll[nb][s] = kb;
                    ncoll[nb]++;
                }
            }
        }
    }
};

}  // namespace

Plan build_plan(const double* cell, int n, const double* pos, int n_digits, int n_per_leaf, int nz,
                const double* bloch, PointOps* points) {
    if (n <= 0) throw std::invalid_argument("number of points must be positive");
    if (n_per_leaf <= 0) throw std::invalid_argument("n_per_leaf must be positive");
    if (nz <= 0) throw std::invalid_argument("nz must be positive (the automatic rc choice is not supported)");
    Plan P;
    P.n_digits_user = n_digits;
    P.dp = digit_params(n_digits);
    P.n_per_leaf = n_per_leaf;
    P.nz = nz;
    P.p = P.dp.n_order;
    P.n_pw = P.dp.n_pw;
    P.n_pw2 = (P.n_pw + 1) / 2;
    P.n_modes = P.n_pw * P.n_pw * P.n_pw2;

    // ---- lattice (avec column-major: avec[j*3+i] = component i of vector j)
    double avec[9];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) avec[j * 3 + i] = cell[j * 3 + i];
    lattice_setup(avec, P.umat, P.qmat);
    if (!(P.umat[0] > 0 && P.umat[4] > 0 && P.umat[8] > 0)) throw std::invalid_argument("degenerate cell");
    utri_inv(P.umat, P.umatinv);
    P.volume = P.umat[0] * P.umat[4] * P.umat[8];
    P.rc = std::min(P.umat[0], std::min(P.umat[4], P.umat[8])) / nz;
    compute_grid(P.umat, P.rc, P.mgrid, P.xgrid0);

    // ---- rotate positions into the umat frame (periodic_dmk.cpp:102-115)
    P.n_src = n;
    P.r_user.resize(3 * (size_t)n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += P.qmat[k + j * 3] * pos[3 * (size_t)i + k];
            P.r_user[3 * (size_t)i + j] = s;
        }

    HostPoints host_points;
    PointOps& ops = points ? *points : host_points;
    ops.load(n, P.r_user.data());
    {
        std::vector<std::array<double, 3>> shifts;
        double lo_ext[3], hi_ext[3];
        image_shifts(P.umat, P.rc, P.mgrid, P.xgrid0, shifts, lo_ext, hi_ext);
        P.img_src_idx = ops.add_images(shifts, lo_ext, hi_ext);
    }
    const int nsall = n + (int)P.img_src_idx.size();
    P.n_all = nsall;

    // ---- level-0 rectangular grid
    const double rc = P.rc;
    int mle[3];
    double xelo[3];
    for (int i = 0; i < 3; ++i) {
        mle[i] = P.mgrid[i] + 2;
        xelo[i] = P.xgrid0[i] - rc;
    }
    const int nb0 = mle[0] * mle[1] * mle[2];
    P.nboxes0 = nb0;
    Builder B;
    for (int iz = 0; iz < mle[2]; ++iz)
        for (int iy = 0; iy < mle[1]; ++iy)
            for (int ix = 0; ix < mle[0]; ++ix) {
                const int b = B.add_box(0, -1);
                B.cen[3 * b + 0] = xelo[0] + (ix + 0.5) * rc;
                B.cen[3 * b + 1] = xelo[1] + (iy + 0.5) * rc;
                B.cen[3 * b + 2] = xelo[2] + (iz + 0.5) * rc;
                int id = 0;
                for (int kz = -1; kz <= 1; ++kz)
                    for (int ky = -1; ky <= 1; ++ky)
                        for (int kx = -1; kx <= 1; ++kx, ++id) {
                            const int jx = ix + kx, jy = iy + ky, jz = iz + kz;
                            if (jx < 0 || jx >= mle[0] || jy < 0 || jy >= mle[1] || jz < 0 || jz >= mle[2])
                                continue;
                            B.coll[b][id] = jz * mle[0] * mle[1] + jy * mle[0] + jx;
                            B.ncoll[b]++;
                        }
            }

    // ---- stable counting sort into level-0 boxes (bin index truncation as
    // the reference: (int)((x - xelo) / rc) clamped to the grid)
    B.ops = &ops;
    for (int s = 0; s < 2; ++s) {
        const std::vector<int> ip = ops.bin0(s, xelo, 1.0 / rc, mle);
        std::vector<int>& se = s == 0 ? B.sse : B.tse;
        for (int b = 0; b < nb0; ++b) {
            se[2 * b] = ip[b];
            se[2 * b + 1] = ip[b + 1] - 1;
        }
    }

    // ---- top-down refinement
    double npl_alpha = 1.5;
    if (const char* s = std::getenv("DMK_NPL_ALPHA")) npl_alpha = std::atof(s);
    const int ndiv = (int)std::ceil(n_per_leaf * npl_alpha);
    int max_level = 0;
    for (int level = 0; level < 50; ++level) {
        bool any = false;
        std::vector<int> at;
        for (int b = 0; b < B.nbox(); ++b)
            if (B.depth[b] == level && B.nchild[b] == 0) at.push_back(b);
        for (int b : at) {
            if (B.scount(b) <= ndiv) continue;
            any = true;
            B.split(b, level, rc);
        }
        B.flush();
        if (!any) break;
        max_level = level + 1;
        const double child_bs = rc / (double)(1 << (level + 1));
        for (int b = 0; b < B.nbox(); ++b)
            if (B.depth[b] == level + 1) B.child_colleagues(b, child_bs);
    }

    // ---- 2:1 balance: a leaf must not touch a non-leaf box two levels finer
    {
        bool changed = true;
        int iter = 0;
        while (changed && iter++ < 50) {
            changed = false;
            for (int L = 0; L <= max_level; ++L) {
                B.flush();  // counts of the boxes split at the previous level
                const double lvl_bs = rc / (double)(1 << L);
                const double child_bs = rc / (double)(1 << (L + 1));
                const double adj_tol = 1.05 * 0.5 * (lvl_bs + child_bs);
                std::vector<int> leaves;
                for (int b = 0; b < B.nbox(); ++b)
                    if (B.depth[b] == L && B.nchild[b] == 0 && B.scount(b) > 0) leaves.push_back(b);
                for (int b : leaves) {
                    if (B.nchild[b] != 0) continue;
                    bool violate = false;
                    for (int ic = 0; ic < 27 && !violate; ++ic) {
                        const int cc = B.coll[b][ic];
                        if (cc < 0 || cc == b || B.nchild[cc] == 0) continue;
                        for (int jc = 0; jc < 8; ++jc) {
                            const int gc = B.children[cc][jc];
                            if (gc < 0 || B.nchild[gc] == 0) continue;
                            bool adj = true;
                            for (int d = 0; d < 3; ++d)
                                if (std::abs(B.cen[3 * b + d] - B.cen[3 * gc + d]) > adj_tol) {
                                    adj = false;
                                    break;
                                }
                            if (adj) {
                                violate = true;
                                break;
                            }
                        }
                    }
                    if (!violate) continue;
                    B.split(b, L, rc);
                    for (int c = 0; c < 8; ++c) B.child_colleagues(B.children[b][c], child_bs);
                    // Make existing boxes list the new children at the mirror
                    // stencil position.
                    for (int c = 0; c < 8; ++c) {
                        const int nb = B.children[b][c];
                        for (int ic = 0; ic < 27; ++ic) {
                            const int kb = B.coll[nb][ic];
                            if (kb < 0 || kb == nb) continue;
                            int s = 0, st = 1;
                            for (int d = 0; d < 3; ++d) {
                                const int di = (int)std::round((B.cen[3 * nb + d] - B.cen[3 * kb + d]) / child_bs);
                                s += (di + 1) * st;
                                st *= 3;
                            }
                            if (s >= 0 && s < 27 && B.coll[kb][s] != nb) {
                                if (B.coll[kb][s] < 0) B.ncoll[kb]++;
                                B.coll[kb][s] = nb;
                            }
                        }
                    }
                    changed = true;
                    if (L + 1 > max_level) max_level = L + 1;
                }
            }
        }
    }

    B.flush();

    // ---- finalize topology
    const int nb = B.nbox();
    P.nboxes = nb;
    P.nlevels = max_level + 1;
    P.depth = B.depth;
    P.parent = B.parent;
    P.nchild = B.nchild;
    P.children = B.children;
    P.colleagues = B.coll;
    P.centers = B.cen;
    P.level_boxes.assign(P.nlevels, {});
    for (int b = 0; b < nb; ++b) P.level_boxes[P.depth[b]].push_back(b);
    P.boxsize.assign(P.nlevels + 1, 0.0);
    P.boxsize[0] = rc;
    for (int l = 1; l <= P.nlevels; ++l) P.boxsize[l] = P.boxsize[l - 1] / 2.0;
    P.is_leaf.assign(nb, 0);
    for (int b = 0; b < nb; ++b) P.is_leaf[b] = (P.nchild[b] == 0);
    P.src_start.resize(nb);
    P.trg_start.resize(nb);
    P.src_count.assign(nb, 0);
    P.trg_count.assign(nb, 0);
    for (int b = 0; b < nb; ++b) {
        P.src_start[b] = B.sse[2 * b];
        P.trg_start[b] = B.tse[2 * b];
        if (P.is_leaf[b]) {
            P.src_count[b] = std::max(0, B.scount(b));
            P.trg_count[b] = std::max(0, B.tcount(b));
        }
    }
    for (int l = P.nlevels - 1; l >= 0; --l)
        for (int b : P.level_boxes[l]) {
            const int dad = P.parent[b];
            if (dad >= 0) {
                P.src_count[dad] += P.src_count[b];
                P.trg_count[dad] += P.trg_count[b];
            }
        }
    // Every point must sit inside its leaf (the reference logs "misplaced
    // particles" otherwise, pbc_tree.cpp:699-732); treat it as a hard error.
    // Inside each leaf, the points are then ordered along a Morton curve of
    // the leaf box: consecutive points (one GPU warp's targets, one chunk of
    // sources) then cover a compact sub-box, so the cutoff tests of the near
    // field agree across a warp.  Sums over a leaf do not depend on the order.
    {
        std::vector<PointOps::Leaf> inside, ls, lt;
        for (int b = 0; b < nb; ++b) {
            if (!P.is_leaf[b]) continue;
            const double* c = &P.centers[3 * b];
            const double h = P.boxsize[P.depth[b]] / 2.0;
            inside.push_back({P.src_start[b], P.src_count[b], {c[0], c[1], c[2]}, h * 1.01});
            if (P.src_count[b] > 1) ls.push_back({P.src_start[b], P.src_count[b], {c[0], c[1], c[2]}, h});
            if (P.trg_count[b] > 1) lt.push_back({P.trg_start[b], P.trg_count[b], {c[0], c[1], c[2]}, h});
        }
        if (ops.outside(0, inside) > 0)
            throw std::invalid_argument("point outside the cell's covering grid (positions must lie in the cell)");
        ops.morton(0, ls);
        ops.morton(1, lt);
    }
    ops.fetch(0, P.src_sorted, P.src_perm);
    ops.fetch(1, P.trg_sorted, P.trg_perm);
    P.src_charge_idx.resize(nsall);
    for (int i = 0; i < nsall; ++i) {
        const int j = P.src_perm[i];
        P.src_charge_idx[i] = j < n ? j : P.img_src_idx[j - n];
    }

    // ---- proxy expansion flags (pbc_tree.cpp:776-811)
    P.ifpwexp.assign(nb, 0);
    for (int b : P.level_boxes[0]) P.ifpwexp[b] = 1;
    for (int l = 1; l < P.nlevels; ++l)
        for (int b : P.level_boxes[l]) {
            if (P.nchild[b] > 0) {
                P.ifpwexp[b] = 1;
                continue;
            }
            for (int ic = 0; ic < 27; ++ic) {
                const int nbx = P.colleagues[b][ic];
                if (nbx >= 0 && P.nchild[nbx] > 0) {
                    P.ifpwexp[b] = 1;
                    break;
                }
            }
        }
    for (int b = 0; b < nb; ++b)
        if (P.src_count[b] == 0 && P.trg_count[b] == 0) P.ifpwexp[b] = 0;
    P.iftensprodeval.assign(nb, 0);
    for (int b = 0; b < nb; ++b)
        if (P.is_leaf[b] && P.src_count[b] + P.trg_count[b] > 0) P.iftensprodeval[b] = 1;

    // ---- near-field list: leaf colleagues, close leaf children of non-leaf
    // colleagues, and close leaf colleagues of the parent (pbc_tree.cpp:851-907)
    std::vector<std::vector<int>> l1(nb);
    for (int l = 0; l < P.nlevels; ++l)
        for (int box : P.level_boxes[l]) {
            if (!P.is_leaf[box]) continue;
            auto& L1 = l1[box];
            const double* cb = &P.centers[3 * box];
            for (int ic = 0; ic < 27; ++ic) {
                const int nbx = P.colleagues[box][ic];
                if (nbx < 0) continue;
                if (P.is_leaf[nbx] && P.src_count[nbx] > 0) {
                    L1.push_back(nbx);
                } else if (P.nchild[nbx] > 0 && l + 1 < P.nlevels) {
                    const double cut = 1.05 * 0.75 * P.boxsize[l];
                    for (int jc = 0; jc < 8; ++jc) {
                        const int kb = P.children[nbx][jc];
                        if (kb < 0 || P.src_count[kb] == 0 || !P.is_leaf[kb]) continue;
                        bool in = true;
                        for (int d = 0; d < 3; ++d)
                            if (std::abs(cb[d] - P.centers[3 * kb + d]) > cut) {
                                in = false;
                                break;
                            }
                        if (in) L1.push_back(kb);
                    }
                }
            }
            if (l == 0) continue;
            const int dad = P.parent[box];
            const double cut2 = 1.5 * 1.05 * P.boxsize[l];
            for (int ic = 0; ic < 27; ++ic) {
                const int nbx = P.colleagues[dad][ic];
                if (nbx < 0 || !P.is_leaf[nbx] || P.src_count[nbx] == 0) continue;
                bool in = true;
                for (int d = 0; d < 3; ++d)
                    if (std::abs(cb[d] - P.centers[3 * nbx + d]) > cut2) {
                        in = false;
                        break;
                    }
                if (in) L1.push_back(nbx);
            }
        }
    P.list1_start.assign(nb + 1, 0);
    for (int b = 0; b < nb; ++b) P.list1_start[b + 1] = P.list1_start[b] + (int)l1[b].size();
    P.list1.reserve(P.list1_start[nb]);
    for (int b = 0; b < nb; ++b) P.list1.insert(P.list1.end(), l1[b].begin(), l1[b].end());

    // ---- upward work (pbc_tree.cpp:909-941)
    P.has_proxy_from_children.assign(nb, 0);
    for (int l = P.nlevels - 1; l >= 0; --l)
        for (int b : P.level_boxes[l]) {
            if (!P.ifpwexp[b] || P.src_count[b] == 0) continue;
            bool child_has = false;
            for (int c = 0; c < 8; ++c) {
                const int ch = P.children[b][c];
                if (ch >= 0 && P.ifpwexp[ch] && P.src_count[ch] > 0) {
                    child_has = true;
                    break;
                }
            }
            if (child_has) {
                P.has_proxy_from_children[b] = 1;
                for (int c = 0; c < 8; ++c) {
                    const int ch = P.children[b][c];
                    if (ch >= 0 && P.src_count[ch] > 0 && !P.ifpwexp[ch]) P.c2proxy_work.push_back({ch, b, l});
                }
            } else {
                P.c2proxy_work.push_back({b, b, l});
            }
        }
    // ---- near-field work: leaves with a list and points, largest first
    for (int b = 0; b < nb; ++b) {
        if (!P.is_leaf[b] || P.list1_start[b + 1] == P.list1_start[b]) continue;
        if (P.src_count[b] == 0 && P.trg_count[b] == 0) continue;
        P.direct_work.push_back(b);
    }
    std::stable_sort(P.direct_work.begin(), P.direct_work.end(), [&](int a, int b) {
        return P.src_count[a] + P.trg_count[a] > P.src_count[b] + P.trg_count[b];
    });

    // ---- storage offsets (pbc_tree.cpp:961-1011)
    const int64_t ncoef = (int64_t)P.p * P.p * P.p;
    P.proxy_up_off.assign(nb, -1);
    P.proxy_down_off.assign(nb, -1);
    P.pw_off.assign(nb, -1);
    for (int b = 0; b < nb; ++b) {
        if (P.ifpwexp[b] && P.src_count[b] > 0) {
            P.proxy_up_off[b] = P.n_proxy_up * ncoef;
            P.n_proxy_up++;
            P.pw_off[b] = P.n_pw_exp * (int64_t)P.n_modes;
            P.n_pw_exp++;
        }
        if ((P.ifpwexp[b] || P.iftensprodeval[b]) && P.src_count[b] + P.trg_count[b] > 0) {
            P.proxy_down_off[b] = P.n_proxy_down * ncoef;
            P.n_proxy_down++;
        }
    }

    if (bloch) {
        for (int d = 0; d < 3; ++d)
            if (!std::isfinite(bloch[d])) throw std::invalid_argument("bloch must be finite");
        P.qp = true;
        for (int d = 0; d < 3; ++d) P.bloch[d] = bloch[d];
    }
    build_tables(P);
    return P;
}

std::string Plan::summary() const {
    std::ostringstream os;
    os << "N=" << n_src << " n_all=" << n_all << " boxes=" << nboxes << " levels=" << nlevels << " (";
    for (int l = 0; l < nlevels; ++l) os << (l ? "/" : "") << level_boxes[l].size();
    int nleaf_t = 0;
    for (int b = 0; b < nboxes; ++b)
        if (is_leaf[b] && trg_count[b] > 0) nleaf_t++;
    os << ") target_leaves=" << nleaf_t << " p=" << p << " n_pw=" << n_pw << " rc=" << rc << " far modes=" << ms
       << "x" << mt << "x" << mu << " pw_boxes=" << n_pw_exp << " c2proxy_work=" << c2proxy_work.size();
    return os.str();
}

}  // namespace pdmkb
