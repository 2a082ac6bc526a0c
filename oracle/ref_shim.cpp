// Checker shim (test infrastructure): C entry points over the reference's own
// standalone sources, compiled from where they lie (cpp/src/dmk/prolate.cpp,
// cpp/src/dmk/legeexps.cpp, cpp/include/dmk/pbc.hpp,
// cpp/include/pdmk/image_layout.hpp) into oracle/_ref/libref.so by
// `make -C oracle ref`.  Used only to generate and check golden fixtures.
#include <dmk/pbc.hpp>
#include <dmk/legeexps.hpp>
#include <dmk/prolate0_fun.hpp>
#include <pdmk/image_layout.hpp>

#include <vector>

extern "C" {

// psi_0^beta at nx points plus the reference's moments (c0, c1, c2, c4).
int ref_pswf(double beta, int nx, const double* x, double* psi, double* intvals4) {
    dmk::Prolate0Fun pf(beta, 10000);
    for (int i = 0; i < nx; ++i) psi[i] = pf.eval_val(x[i]);
    auto c = pf.intvals(beta);
    for (int i = 0; i < 4; ++i) intvals4[i] = c[i];
    return 0;
}

// Gauss-Legendre rule of the reference (legerts).
int ref_legendre(int n, double* x, double* w) {
    dmk::legerts(1, n, x, w);
    return 0;
}

// Lattice QR, grid and image layout of the reference for 3D (positions are
// Cartesian, rotated here as the reference does): returns the number
// of images; fills umat/qmat (9 each), mgrid (3), xgrid0 (3), and, if
// img_idx != nullptr, the originating source index of each image (capacity cap).
long ref_images(const double* avec, double rc_nz, int n, const double* pos, double* umat, double* qmat,
                int* mgrid, double* xgrid0, double* rc_out, int* img_idx, long cap) {
    dmk::pbc::lattice_setup<double, 3>(avec, umat, qmat);
    // rotation into the umat frame as the reference's tree constructor does
    std::vector<double> pos_rotated(3 * (size_t)n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += qmat[k + j * 3] * pos[3 * (size_t)i + k];
            pos_rotated[3 * (size_t)i + j] = s;
        }
    double rc = std::min(umat[0], std::min(umat[4], umat[8])) / rc_nz;
    *rc_out = rc;
    dmk::pbc::compute_grid<double, 3>(umat, rc, mgrid, xgrid0);
    std::vector<double> img;
    std::vector<int> idx;
    pdmk::generate_images_with_src_idx<double, 3>(umat, rc, mgrid, xgrid0, n, pos_rotated.data(), img, idx);
    if (img_idx)
        for (long i = 0; i < (long)idx.size() && i < cap; ++i) img_idx[i] = idx[i];
    return (long)idx.size();
}
}
