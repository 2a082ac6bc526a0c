// Host-side "plan" for one periodic DMK tree: geometry, the adaptive tree over
// originals + lattice images, interaction/work lists and every precomputed
// table the evaluate path needs.  It is built once per tree on the host (the
// reference's PeriodicDMKTreeT::Impl constructor, cpp/src/periodic_dmk.cpp:41-139,
// plus the PBCTree constructor, cpp/src/dmk/pbc_tree.cpp:138-770) and then
// flattened and uploaded to the GPU once.
//
// Conventions follow the reference:
//   * cell[j*3+i] = component i of lattice vector j.
//   * umat / qmat are 3x3 column-major (m[i + 3*j]).
//   * proxy coefficients are (p,p,p) with x fastest; plane-wave expansions are
//     (n,n,n2) complex with the x frequency fastest and the half-space axis z.
#pragma once
#include <array>
#include <complex>
#include <cstdint>
#include <string>
#include <vector>

namespace pdmkb {

using cplx = std::complex<double>;

// Expansion parameters selected from eps (cpp/src/dmk/util.cpp:12-37,
// cpp/include/dmk/tree.hpp:17-90, cpp/src/dmk/pbc_tree.cpp:148).
struct DigitParams {
    int n_digits_tree;  // round(log10(1/eps) - 0.1), selects the residual polynomial
    double eps;
    double beta;
    int n_order;  // p
    int n_pw;     // n (odd)
};
DigitParams digit_params(int n_digits_user);

// Monomial coefficients of the residual polynomial P(x), x = (r - b/2) * 2/b,
// R_b(r) = P(x)/r for r < b (cpp/src/dmk/aot_kernels.cpp:229-317, selected as
// in :320-456).
const std::vector<double>& residual_coeffs(int n_digits_tree);

struct C2PWork {
    int src_box;
    int center_box;
    int level;
};

struct LevelTables {
    double hpw = 0;                 // plane-wave spacing of this level's difference kernel
    std::vector<cplx> poly2pw;      // n x p, column-major: poly2pw[k + n*a]
    std::vector<cplx> pw2poly;      // n x p, column-major
    std::vector<double> radialft;   // n*n*n2 real, tensor-product layout
    std::vector<double> shift;      // 27 stencils x (M re | M im), kernel FT fused in
};

struct Plan {
    // ---- parameters
    int n_digits_user = 6;
    DigitParams dp{};
    int n_per_leaf = 300, nz = 4;
    int p = 0, n_pw = 0, n_pw2 = 0, n_modes = 0;  // n_modes = n*n*n2
    double rc = 0;
    double umat[9]{}, qmat[9]{}, umatinv[9]{};
    int mgrid[3]{};
    double xgrid0[3]{};
    double volume = 0;

    // ---- points
    int n_src = 0;  // N originals (also the targets)
    int n_all = 0;  // originals + images
    std::vector<double> r_user;        // 3N rotated positions, user order
    std::vector<int> img_src_idx;      // image j -> originating user index
    std::vector<double> src_sorted;    // 3*n_all
    std::vector<int> src_charge_idx;   // sorted source -> user charge index
    std::vector<int> src_perm;         // sorted source -> index in (originals ++ images)
    std::vector<double> trg_sorted;    // 3*N
    std::vector<int> trg_perm;         // sorted target -> user index

    // ---- boxes
    int nboxes = 0, nlevels = 0, nboxes0 = 0;
    std::vector<int> depth, parent, nchild;
    std::vector<std::array<int, 8>> children;
    std::vector<std::array<int, 27>> colleagues;
    std::vector<double> centers;  // 3*nboxes
    std::vector<int> src_start, src_count, trg_start, trg_count;  // counts are subtree sums
    std::vector<uint8_t> is_leaf, ifpwexp, iftensprodeval, has_proxy_from_children;
    std::vector<std::vector<int>> level_boxes;
    std::vector<double> boxsize;  // nlevels + 1
    std::vector<int64_t> proxy_up_off, proxy_down_off, pw_off;  // element offsets, -1 = none
    int64_t n_proxy_up = 0, n_proxy_down = 0, n_pw_exp = 0;      // number of boxes with storage

    // ---- lists
    std::vector<int> list1_start, list1;  // CSR over boxes (nboxes + 1)
    std::vector<C2PWork> c2proxy_work;
    std::vector<int> direct_work;

    // ---- tables
    std::vector<double> w0;            // self-interaction constant per depth (nlevels + 1)
    std::vector<double> p2c;           // 8 children x 3 dims x (p x p) column-major
    std::vector<LevelTables> lev;      // per level
    std::vector<double> resid;         // residual polynomial coefficients
    double psi0_at_zero = 0, c0 = 0;

    // ---- quasi-periodic evaluation: images at x + R carry e^{i bloch.R}, the
    // Bloch vector taken in the lattice-QR frame of the tree (as the reference's
    // generate_images / far_field_nufft use it, cpp/include/dmk/pbc.hpp:142-256,
    // cpp/src/dmk/pbc.cpp:250-357)
    bool qp = false;
    double bloch[3]{};

    // ---- periodic far field (windowed kernel W_rc)
    int ms = 0, mt = 0, mu = 0;        // mode counts along the three reciprocal axes (|bloch| added when qp)
    std::vector<double> ff_weights;    // ms*mt*mu, ms fastest, modes -m/2 .. (m-1)/2

    std::string summary() const;
};

class PointOps;  // points.hpp

// Build a plan.  cell[j*3+i] = component i of lattice vector j; pos[3*i+d].
// bloch (3 doubles, or null): quasi-periodic plan (see Plan::qp).
// points: where the point-heavy steps run (null: on the host; the GPU form is
// build_plan_device, device/tree_build.cu); the plan does not depend on it.
// Throws std::invalid_argument on bad input.
Plan build_plan(const double* cell, int n, const double* pos, int n_digits, int n_per_leaf, int nz,
                const double* bloch = nullptr, PointOps* points = nullptr);

}  // namespace pdmkb
