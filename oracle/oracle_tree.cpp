// ORACLE — test infrastructure only.  Nothing in the product links, imports or
// calls this file; only tests/ load it, as the checker.
//
// An independent restatement of the reference's tree construction and
// interaction lists, used to check the product's host plan box for box.  It
// shares no code with the product's builder and is written differently:
//   * boxes are keys (level, ix, iy, iz) on the level's grid of side rc/2^level,
//     looked up in a hash map; adjacency is integer arithmetic on the keys
//     (same-level colleagues differ by at most 1 per axis; a box at level L+1
//     touches a box at level L when its index lies in [2I-1, 2I+2] per axis),
//     which is what the reference's centre-distance tolerances select;
//   * points are not partitioned in place: each point descends from its
//     level-0 bin to the box it falls in by the octant rule, and a box's points
//     are the points that reach it, in input order (the reference's stable
//     partitions keep input order inside every box);
//   * the 2:1 balance is computed as the least fixed point of its refinement
//     rule: repeat until no leaf with sources touches a non-leaf box two
//     levels finer.
// Rules restated (reference file:line):
//   lattice QR, grid, rc                 cpp/include/dmk/pbc.hpp:23-117, cpp/src/periodic_dmk.cpp:62-81
//   rotation into the QR frame, images   cpp/src/periodic_dmk.cpp:102-136, cpp/include/pdmk/image_layout.hpp:14-88
//   level-0 bins (truncation, clamp)     cpp/include/dmk/pbc.hpp:344-391
//   refinement (> ceil(1.5 npl), >= centre, child centre = parent +- rc/2^(L+2))
//                                        cpp/src/dmk/pbc_tree.cpp:60-136,299-428
//   2:1 balance                          cpp/src/dmk/pbc_tree.cpp:438-598
//   ifpwexp / list1 / charge-to-proxy work / direct work
//                                        cpp/src/dmk/pbc_tree.cpp:776-959
//   near-field cutoff b per list entry   cpp/src/dmk/pbc_tree.cpp:1503-1514
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include "../periodicdmk_b200/csrc/host/plan.hpp"

namespace {

struct Key {
    int l, x, y, z;
    bool operator==(const Key& o) const { return l == o.l && x == o.x && y == o.y && z == o.z; }
};
struct KeyHash {
    size_t operator()(const Key& k) const {
        uint64_t h = (uint64_t)(uint32_t)k.l * 0x9E3779B97F4A7C15ULL;
        h ^= (uint64_t)(uint32_t)k.x * 0xC2B2AE3D27D4EB4FULL + (h << 6) + (h >> 2);
        h ^= (uint64_t)(uint32_t)k.y * 0x165667B19E3779F9ULL + (h << 6) + (h >> 2);
        h ^= (uint64_t)(uint32_t)k.z * 0x27D4EB2F165667C5ULL + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};
bool key_less(const Key& a, const Key& b) {
    if (a.l != b.l) return a.l < b.l;
    if (a.z != b.z) return a.z < b.z;
    if (a.y != b.y) return a.y < b.y;
    return a.x < b.x;
}

struct OBox {
    Key k;
    double c[3];
    int parent = -1;
    int child[8];  // child index = octant bits (x, y, z) -> -1 if none
    bool leaf = true;
    std::vector<int> src, trg;  // point indices (sources: originals ++ images)
    int nsrc = 0, ntrg = 0;     // subtree counts
};

struct OTree {
    double rc = 0, umat[9], qmat[9];
    int mgrid[3], mle[3];
    double xgrid0[3], xelo[3];
    int n = 0, nall = 0;
    std::vector<double> pts;   // 3 * nall: rotated originals, then images
    std::vector<OBox> box;
    std::unordered_map<Key, int, KeyHash> find;
    int nlev = 0;
    std::vector<double> bs;    // box size per level (+1 extra)
    std::vector<uint8_t> pwexp;

    int lookup(const Key& k) const {
        auto it = find.find(k);
        return it == find.end() ? -1 : it->second;
    }
};

// Modified Gram-Schmidt QR of the lattice with columns sorted by length
// (longest first); umat upper triangular, qmat orthogonal (column-major).
void qr_lattice(const double* a, double* u, double* q) {
    int ord[3] = {0, 1, 2};
    double len[3];
    for (int j = 0; j < 3; ++j) len[j] = std::sqrt(a[3 * j] * a[3 * j] + a[3 * j + 1] * a[3 * j + 1] + a[3 * j + 2] * a[3 * j + 2]);
    // selection order of the reference: for i < j, swap when len[j] > len[i]
    for (int i = 0; i < 2; ++i)
        for (int j = i + 1; j < 3; ++j)
            if (len[j] > len[i]) {
                std::swap(len[i], len[j]);
                std::swap(ord[i], ord[j]);
            }
    double col[3][3];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) col[j][i] = a[3 * ord[j] + i];
    std::memset(u, 0, 9 * sizeof(double));
    double e[3][3];
    for (int i = 0; i < 3; ++i) e[0][i] = col[0][i] / len[0];
    u[0] = len[0];
    for (int j = 1; j < 3; ++j) {
        double v[3] = {col[j][0], col[j][1], col[j][2]};
        double r[2] = {0, 0};
        for (int k = 0; k < j; ++k) {
            double d = 0;
            for (int i = 0; i < 3; ++i) d += e[k][i] * col[j][i];
            r[k] = d;
        }
        for (int i = 0; i < 3; ++i) {
            double t = col[j][i];
            for (int k = 0; k < j; ++k) t -= r[k] * e[k][i];
            v[i] = t;
        }
        double nv = 0;
        for (int i = 0; i < 3; ++i) nv += v[i] * v[i];
        nv = std::sqrt(nv);
        for (int i = 0; i < 3; ++i) e[j][i] = v[i] / nv;
        for (int k = 0; k < j; ++k) u[k + 3 * j] = r[k];
        u[j + 3 * j] = nv;
    }
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) q[i + 3 * j] = e[j][i];
}

void build_geometry(OTree& T, const double* cell, int n, const double* pos, int nz) {
    qr_lattice(cell, T.umat, T.qmat);
    T.rc = std::min(T.umat[0], std::min(T.umat[4], T.umat[8])) / nz;
    for (int i = 2; i >= 0; --i) {
        double lo = 0, hi = T.umat[i + 3 * i];
        for (int j = i + 1; j < 3; ++j) {
            lo += std::min(0.0, T.umat[i + 3 * j]);
            hi += std::max(0.0, T.umat[i + 3 * j]);
        }
        T.mgrid[i] = std::max(1, (int)std::ceil((hi - lo) / T.rc));
        T.xgrid0[i] = lo;
    }
    T.n = n;
    T.pts.resize(3 * (size_t)n);
    for (int p = 0; p < n; ++p)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += T.qmat[k + 3 * j] * pos[3 * (size_t)p + k];
            T.pts[3 * (size_t)p + j] = s;
        }
    // lattice images inside the extended grid, in the reference's shift order
    const double* U = T.umat;
    double elo[3], ehi[3], blo[3], bhi[3];
    for (int i = 0; i < 3; ++i) {
        elo[i] = T.xgrid0[i] - T.rc;
        ehi[i] = T.xgrid0[i] + (T.mgrid[i] + 1) * T.rc;
        blo[i] = T.xgrid0[i];
        double w = U[i + 3 * i];
        for (int j = i + 1; j < 3; ++j) w += std::abs(U[i + 3 * j]);
        bhi[i] = T.xgrid0[i] + w;
    }
    const int m3 = (int)((T.mgrid[2] + 1) * T.rc / U[8]) + 1;
    for (int k3 = -m3; k3 <= m3; ++k3) {
        const double s3 = U[8] * k3;
        if (blo[2] + s3 > ehi[2] || bhi[2] + s3 < elo[2]) continue;
        const int m2 = (int)(((T.mgrid[1] + 1) * T.rc + std::abs(U[7] * k3)) / U[4]) + 1;
        for (int k2 = -m2; k2 <= m2; ++k2) {
            const double s2 = U[4] * k2 + U[7] * k3;
            if (blo[1] + s2 > ehi[1] || bhi[1] + s2 < elo[1]) continue;
            const double o1 = U[3] * k2 + U[6] * k3;
            const int m1 = (int)(((T.mgrid[0] + 1) * T.rc + std::abs(o1)) / U[0]) + 1;
            for (int k1 = -m1; k1 <= m1; ++k1) {
                if (!k1 && !k2 && !k3) continue;
                const double s1 = U[0] * k1 + o1;
                if (blo[0] + s1 > ehi[0] || bhi[0] + s1 < elo[0]) continue;
                for (int p = 0; p < n; ++p) {
                    const double x = T.pts[3 * (size_t)p] + s1, y = T.pts[3 * (size_t)p + 1] + s2,
                                 z = T.pts[3 * (size_t)p + 2] + s3;
                    if (x < elo[0] || x > ehi[0] || y < elo[1] || y > ehi[1] || z < elo[2] || z > ehi[2]) continue;
                    T.pts.push_back(x);
                    T.pts.push_back(y);
                    T.pts.push_back(z);
                }
            }
        }
    }
    T.nall = (int)(T.pts.size() / 3);
}

int new_box(OTree& T, const Key& k, int parent) {
    OBox b;
    b.k = k;
    b.parent = parent;
    std::fill(b.child, b.child + 8, -1);
    T.box.push_back(std::move(b));
    const int id = (int)T.box.size() - 1;
    T.find[k] = id;
    return id;
}

// Split box b into 8 children; its points (sources and targets, in order)
// go to the child of their octant (coordinate >= centre -> upper half).
void split(OTree& T, int b) {
    const int L = T.box[b].k.l;
    const double half = T.rc / std::ldexp(1.0, L + 2);
    T.box[b].leaf = false;
    for (int o = 0; o < 8; ++o) {
        const Key& pk = T.box[b].k;
        const Key k{L + 1, 2 * pk.x + (o & 1), 2 * pk.y + ((o >> 1) & 1), 2 * pk.z + ((o >> 2) & 1)};
        const int c = new_box(T, k, b);
        for (int d = 0; d < 3; ++d) T.box[c].c[d] = T.box[b].c[d] + (((o >> d) & 1) ? half : -half);
        T.box[b].child[o] = c;
    }
    auto octant = [&](const double* x) {
        int o = 0;
        for (int d = 0; d < 3; ++d)
            if (x[d] >= T.box[b].c[d]) o |= 1 << d;
        return o;
    };
    for (int p : T.box[b].src) T.box[T.box[b].child[octant(&T.pts[3 * (size_t)p])]].src.push_back(p);
    for (int p : T.box[b].trg) T.box[T.box[b].child[octant(&T.pts[3 * (size_t)p])]].trg.push_back(p);
    T.box[b].src.clear();
    T.box[b].src.shrink_to_fit();
    T.box[b].trg.clear();
    T.box[b].trg.shrink_to_fit();
}

void build_tree(OTree& T, int npl) {
    for (int i = 0; i < 3; ++i) {
        T.mle[i] = T.mgrid[i] + 2;
        T.xelo[i] = T.xgrid0[i] - T.rc;
    }
    for (int z = 0; z < T.mle[2]; ++z)
        for (int y = 0; y < T.mle[1]; ++y)
            for (int x = 0; x < T.mle[0]; ++x) {
                const int b = new_box(T, Key{0, x, y, z}, -1);
                const int ii[3] = {x, y, z};
                for (int d = 0; d < 3; ++d) T.box[b].c[d] = T.xelo[d] + (ii[d] + 0.5) * T.rc;
            }
    auto bin0 = [&](const double* p) {
        int ii[3];
        for (int d = 0; d < 3; ++d) {
            int v = (int)((p[d] - T.xelo[d]) * (1.0 / T.rc));
            ii[d] = std::min(std::max(v, 0), T.mle[d] - 1);
        }
        return (ii[2] * T.mle[1] + ii[1]) * T.mle[0] + ii[0];
    };
    for (int p = 0; p < T.nall; ++p) T.box[bin0(&T.pts[3 * (size_t)p])].src.push_back(p);
    for (int p = 0; p < T.n; ++p) T.box[bin0(&T.pts[3 * (size_t)p])].trg.push_back(p);
    // refinement by levels
    const char* sa = std::getenv("DMK_NPL_ALPHA");
    const int limit = (int)std::ceil(npl * (sa ? std::atof(sa) : 1.5));
    int deepest = 0;
    for (int L = 0; L < 50; ++L) {
        std::vector<int> todo;
        for (int b = 0; b < (int)T.box.size(); ++b)
            if (T.box[b].k.l == L && T.box[b].leaf && (int)T.box[b].src.size() > limit) todo.push_back(b);
        if (todo.empty()) break;
        for (int b : todo) split(T, b);
        deepest = L + 1;
    }
    // 2:1 balance: least fixed point of "a leaf with sources that touches a
    // non-leaf box two levels finer is split"
    auto touches_fine_nonleaf = [&](int b) {
        const Key k = T.box[b].k;
        for (int z = 2 * k.z - 1; z <= 2 * k.z + 2; ++z)
            for (int y = 2 * k.y - 1; y <= 2 * k.y + 2; ++y)
                for (int x = 2 * k.x - 1; x <= 2 * k.x + 2; ++x) {
                    const int g = T.lookup(Key{k.l + 1, x, y, z});
                    if (g >= 0 && !T.box[g].leaf && T.box[g].parent != b) return true;
                }
        return false;
    };
    for (bool changed = true; changed;) {
        changed = false;
        const int nb = (int)T.box.size();
        for (int b = 0; b < nb; ++b) {
            if (!T.box[b].leaf || T.box[b].src.empty()) continue;
            if (!touches_fine_nonleaf(b)) continue;
            split(T, b);
            deepest = std::max(deepest, T.box[b].k.l + 1);
            changed = true;
        }
    }
    T.nlev = deepest + 1;
    T.bs.resize(T.nlev + 1);
    T.bs[0] = T.rc;
    for (int l = 1; l <= T.nlev; ++l) T.bs[l] = T.bs[l - 1] / 2;
    // subtree counts, deepest level first
    std::vector<int> order(T.box.size());
    for (int b = 0; b < (int)T.box.size(); ++b) order[b] = b;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return T.box[a].k.l > T.box[c].k.l; });
    for (int b : order) {
        OBox& B = T.box[b];
        if (B.leaf) {
            B.nsrc = (int)B.src.size();
            B.ntrg = (int)B.trg.size();
        }
        if (B.parent >= 0) {
            T.box[B.parent].nsrc += B.nsrc;
            T.box[B.parent].ntrg += B.ntrg;
        }
    }
    // plane-wave expansion flags
    T.pwexp.assign(T.box.size(), 0);
    for (int b = 0; b < (int)T.box.size(); ++b) {
        const OBox& B = T.box[b];
        bool f = B.k.l == 0 || !B.leaf;
        for (int dz = -1; dz <= 1 && !f; ++dz)
            for (int dy = -1; dy <= 1 && !f; ++dy)
                for (int dx = -1; dx <= 1 && !f; ++dx) {
                    const int c = T.lookup(Key{B.k.l, B.k.x + dx, B.k.y + dy, B.k.z + dz});
                    if (c >= 0 && !T.box[c].leaf) f = true;
                }
        T.pwexp[b] = f && (B.nsrc > 0 || B.ntrg > 0);
    }
}

// list1 of leaf b: (box, cutoff b) entries
void near_list(const OTree& T, int b, std::vector<std::pair<int, double>>& out) {
    out.clear();
    const OBox& B = T.box[b];
    const int l = B.k.l;
    auto cutoff = [&](int s) {
        const int sl = T.box[s].k.l;
        if (T.pwexp[s] && s == b) return T.bs[sl] / 2;
        if (sl < l) return T.bs[l];
        return T.bs[sl];
    };
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int c = T.lookup(Key{l, B.k.x + dx, B.k.y + dy, B.k.z + dz});
                if (c < 0) continue;
                if (T.box[c].leaf) {
                    if (T.box[c].nsrc > 0) out.push_back({c, cutoff(c)});
                } else if (l + 1 < T.nlev) {
                    for (int o = 0; o < 8; ++o) {
                        const int g = T.box[c].child[o];
                        if (g < 0 || !T.box[g].leaf || T.box[g].nsrc == 0) continue;
                        const Key& gk = T.box[g].k;
                        if (gk.x >= 2 * B.k.x - 1 && gk.x <= 2 * B.k.x + 2 && gk.y >= 2 * B.k.y - 1 &&
                            gk.y <= 2 * B.k.y + 2 && gk.z >= 2 * B.k.z - 1 && gk.z <= 2 * B.k.z + 2)
                            out.push_back({g, cutoff(g)});
                    }
                }
            }
    if (l == 0 || B.parent < 0) return;
    const Key& pk = T.box[B.parent].k;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const Key ck{pk.l, pk.x + dx, pk.y + dy, pk.z + dz};
                const int c = T.lookup(ck);
                if (c < 0 || !T.box[c].leaf || T.box[c].nsrc == 0) continue;
                if (B.k.x >= 2 * ck.x - 1 && B.k.x <= 2 * ck.x + 2 && B.k.y >= 2 * ck.y - 1 &&
                    B.k.y <= 2 * ck.y + 2 && B.k.z >= 2 * ck.z - 1 && B.k.z <= 2 * ck.z + 2)
                    out.push_back({c, cutoff(c)});
            }
}

// Integer key of a product-plan box from its centre.
Key plan_key(const pdmkb::Plan& P, const double* xelo, int b) {
    const int l = P.depth[b];
    const double h = P.boxsize[l];
    Key k{l, 0, 0, 0};
    int* kk[3] = {&k.x, &k.y, &k.z};
    for (int d = 0; d < 3; ++d) *kk[d] = (int)std::lround((P.centers[3 * b + d] - xelo[d]) / h - 0.5);
    return k;
}

}  // namespace

extern "C" {

// Build the tree with the independent builder above and compare it with the
// product's host plan for the same input.  out[0..15]:
//   0 boxes (oracle)          1 levels (oracle)        2 leaves with sources
//   3 box-set mismatches      4 leaf source-set mismatches
//   5 leaf target-set mismatches 6 plane-wave-flag mismatches
//   7 list1 entry mismatches (box + cutoff)  8 list1 entries (oracle)
//   9 charge-to-proxy work mismatches       10 direct-work mismatches
//   11 image count mismatch (|oracle - plan|) 12 rc/umat mismatch (1 if any)
//   13..15 boxes at levels 0, 1, 2 (oracle)
// Returns 0 on success, -1 on error.
int oracle_tree_compare(const double* cell, int n, const double* pos, int n_digits, int n_per_leaf, int nz,
                        long long* out) {
    try {
        std::memset(out, 0, 16 * sizeof(long long));
        OTree T;
        build_geometry(T, cell, n, pos, nz);
        build_tree(T, n_per_leaf);
        const pdmkb::Plan P = pdmkb::build_plan(cell, n, pos, n_digits, n_per_leaf, nz);
        out[0] = (long long)T.box.size();
        out[1] = T.nlev;
        for (const auto& b : T.box)
            if (b.leaf && b.nsrc > 0) out[2]++;
        out[11] = std::llabs((long long)T.nall - (long long)P.n_all);
        bool geo = std::abs(T.rc - P.rc) > 0;
        for (int i = 0; i < 9; ++i) geo = geo || T.umat[i] != P.umat[i];
        out[12] = geo ? 1 : 0;
        for (const auto& b : T.box)
            if (b.k.l <= 2) out[13 + b.k.l]++;
        // box sets
        std::unordered_map<Key, int, KeyHash> pmap;
        for (int b = 0; b < P.nboxes; ++b) pmap[plan_key(P, T.xelo, b)] = b;
        std::vector<int> o2p(T.box.size(), -1);
        for (int b = 0; b < (int)T.box.size(); ++b) {
            auto it = pmap.find(T.box[b].k);
            if (it == pmap.end()) {
                out[3]++;
                continue;
            }
            o2p[b] = it->second;
            if (P.is_leaf[it->second] != (T.box[b].leaf ? 1 : 0)) out[3]++;
        }
        out[3] += std::llabs((long long)P.nboxes - (long long)T.box.size());
        for (int b = 0; b < (int)T.box.size(); ++b) {
            const int q = o2p[b];
            if (q < 0) continue;
            const OBox& B = T.box[b];
            if ((T.pwexp[b] != 0) != (P.ifpwexp[q] != 0)) out[6]++;
            if (!B.leaf) continue;
            // sources: the plan's sorted range mapped back to point identities
            std::vector<int> ps, pt;
            for (int i = P.src_start[q]; i < P.src_start[q] + P.src_count[q]; ++i) ps.push_back(P.src_perm[i]);
            for (int i = P.trg_start[q]; i < P.trg_start[q] + P.trg_count[q]; ++i) pt.push_back(P.trg_perm[i]);
            std::sort(ps.begin(), ps.end());
            std::sort(pt.begin(), pt.end());
            if (ps != B.src) out[4]++;  // oracle lists are in input order (ascending)
            if (pt != B.trg) out[5]++;
        }
        // list1 of every leaf with sources or targets
        std::vector<std::pair<int, double>> nl;
        for (int b = 0; b < (int)T.box.size(); ++b) {
            const int q = o2p[b];
            if (q < 0 || !T.box[b].leaf) continue;
            near_list(T, b, nl);
            out[8] += (long long)nl.size();
            std::vector<std::pair<Key, double>> a, c;
            for (auto& e : nl) a.push_back({T.box[e.first].k, e.second});
            for (int li = P.list1_start[q]; li < P.list1_start[q + 1]; ++li) {
                const int sb = P.list1[li];
                const int sl = P.depth[sb], tl = P.depth[q];
                double bb = P.boxsize[sl];
                if (P.ifpwexp[sb] && sb == q) bb /= 2;
                else if (sl < tl) bb = P.boxsize[tl];
                c.push_back({plan_key(P, T.xelo, sb), bb});
            }
            auto lt = [](const std::pair<Key, double>& x, const std::pair<Key, double>& y) {
                if (!(x.first == y.first)) return key_less(x.first, y.first);
                return x.second < y.second;
            };
            std::sort(a.begin(), a.end(), lt);
            std::sort(c.begin(), c.end(), lt);
            size_t i = 0, j = 0;
            while (i < a.size() || j < c.size()) {
                if (i < a.size() && j < c.size() && a[i].first == c[j].first && a[i].second == c[j].second) {
                    ++i;
                    ++j;
                } else if (j >= c.size() || (i < a.size() && lt(a[i], c[j]))) {
                    out[7]++;
                    ++i;
                } else {
                    out[7]++;
                    ++j;
                }
            }
        }
        // charge-to-proxy work: (source box, centre box) pairs
        {
            std::vector<std::array<int, 8>> ow, pw;
            for (int b = 0; b < (int)T.box.size(); ++b) {
                const OBox& B = T.box[b];
                if (!T.pwexp[b] || B.nsrc == 0) continue;
                bool from_children = false;
                for (int o = 0; o < 8; ++o) {
                    const int c = B.child[o];
                    if (c >= 0 && T.pwexp[c] && T.box[c].nsrc > 0) from_children = true;
                }
                auto push = [&](int s, int c) {
                    const Key& a = T.box[s].k;
                    const Key& d = T.box[c].k;
                    ow.push_back({a.l, a.x, a.y, a.z, d.l, d.x, d.y, d.z});
                };
                if (!from_children) {
                    push(b, b);
                } else {
                    for (int o = 0; o < 8; ++o) {
                        const int c = B.child[o];
                        if (c >= 0 && T.box[c].nsrc > 0 && !T.pwexp[c]) push(c, b);
                    }
                }
            }
            for (const auto& w : P.c2proxy_work) {
                const Key a = plan_key(P, T.xelo, w.src_box), d = plan_key(P, T.xelo, w.center_box);
                pw.push_back({a.l, a.x, a.y, a.z, d.l, d.x, d.y, d.z});
            }
            std::sort(ow.begin(), ow.end());
            std::sort(pw.begin(), pw.end());
            if (ow != pw) {
                std::vector<std::array<int, 8>> diff;
                std::set_symmetric_difference(ow.begin(), ow.end(), pw.begin(), pw.end(), std::back_inserter(diff));
                out[9] = (long long)diff.size();
            }
        }
        // direct work: leaves with a non-empty list1 and sources or targets
        {
            std::vector<std::array<int, 4>> od, pd;
            for (int b = 0; b < (int)T.box.size(); ++b) {
                const OBox& B = T.box[b];
                if (!B.leaf || (B.nsrc == 0 && B.ntrg == 0)) continue;
                near_list(T, b, nl);
                if (nl.empty()) continue;
                od.push_back({B.k.l, B.k.x, B.k.y, B.k.z});
            }
            for (int q : P.direct_work) {
                const Key k = plan_key(P, T.xelo, q);
                pd.push_back({k.l, k.x, k.y, k.z});
            }
            std::sort(od.begin(), od.end());
            std::sort(pd.begin(), pd.end());
            if (od != pd) {
                std::vector<std::array<int, 4>> diff;
                std::set_symmetric_difference(od.begin(), od.end(), pd.begin(), pd.end(), std::back_inserter(diff));
                out[10] = (long long)diff.size();
            }
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle_tree_compare: %s\n", e.what());
        return -1;
    }
}

}  // extern "C"
